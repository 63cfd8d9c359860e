// Host driver of the 3D update: the reference's Sim3D step sequence in
// throughput mode (two phi pools, two aggregate slots; reference
// src/pf3d/sim.cu:1460-1651):
//
//   snapshot accepted cells -> measure (tumble on, surface on full-moment
//   steps) -> motion -> clear next S -> update -> repair if fatal ->
//   finalize origins -> restore if fatal -> advance step counter.
//
// pfb_sim3d_set_fused(s, 1) runs the measurement, motion and update as one
// fused launch (k_step3d) after the clear; the separate launches stay the
// default, being faster on a B200. Pairs of steps without a surface pass are
// replayed from one CUDA graph.
//
// Cells are visited in the Morton order of their brick centres (the launches'
// selection list, refreshed every kOrderRefresh steps): clusters in flight at
// the same time then touch neighbouring aggregate words, which stay in L2
// across the eight-fold overlap of the bricks. Cells are independent within a
// step, so the order changes no result.
//
// A fresh start seeds tanh spheres with the calibrated radius, builds S from
// them and measures once without a tumble (src/pf3d/sim.cu:1100-1180).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "pfb3d_common.cuh"
#include "pfb_internal.h"

using namespace pfb;
using namespace pfb::p3;

#define PFB3_CU(expr, what)                                                               \
    do {                                                                                  \
        const cudaError_t e_ = (expr);                                                    \
        if (e_ != cudaSuccess) return set_error(PFB_E_CUDA, "%s: %s", what, cudaGetErrorString(e_)); \
    } while (0)
#define PFB3_RC(expr)          \
    do {                       \
        const int r_ = (expr); \
        if (r_) return r_;     \
    } while (0)

struct pfb_sim3d {
    pfb_params3d p{};
    int device = 0;
    int B = 0, N = 0;
    pfb_layout3d L{};
    size_t s_words = 0, cell_words = 0;
    float* d_phi[2] = {nullptr, nullptr};
    uint32_t* d_S[2] = {nullptr, nullptr};
    pfb_cell3d* d_cells = nullptr;
    pfb_cell3d* d_accepted = nullptr;
    uint32_t* d_flags = nullptr;
    uint64_t* d_step = nullptr;
    float* d_wall = nullptr;
    float* d_wall_psi = nullptr;  // channel: psi_w^2 per plane (diagnostics)
    pfb_vec3* d_centres = nullptr;
    cudaStream_t stream = nullptr;
    int cur_phi = 0, cur_S = 0;
    long long steps_done = 0;
    double V0 = 0.0;
    pfb::Boundary3D* bnd = nullptr;  // open PFB3D recorder
    int fused = 0;                   // 1: one fused launch per step
    int* d_order = nullptr;          // visit order of the cells
    bool use_order = true;
    long long order_step = -1;       // step of the last order refresh
    bool use_graph = true;
    cudaGraph_t graph = nullptr;     // two steps from buffer parity 0
    cudaGraphExec_t graph_exec = nullptr;
    // adaptive bricks: cells whose support outgrew B live in their own cubes
    // of edge storage_edge > B; cube[cur_cube][n] holds the current field
    int max_edge = 0;                   // largest cube the domain allows
    std::vector<float*> h_cube[2];      // per cell; null for base cells
    float** d_cube[2] = {nullptr, nullptr};
    std::vector<int> prom_ids;          // promoted cells in id order
    int* d_prom_ids = nullptr;
    int prom_edge = 0;                  // largest promoted edge
    uint32_t* d_requests = nullptr;     // support-exhaustion requests (restore pass)
    long long accepted = 0;             // accepted steps at the last synchronisation
    long long next_compact = 0;         // accepted step of the next compaction
    long long recoveries = 0;
    int cur_cube = 0;                   // current side of the promoted double buffers
    // storage mode (reference StorageMode3D): 0 throughput (two phi pools,
    // two aggregates), 1 balanced (one pool, two aggregates, scratch bricks),
    // 2 compact (one pool, one aggregate rebuilt after every update)
    int mem_mode = 0;
    int mode_request = -1;              // as created: -1 auto
    int slots = 0;                      // scratch bricks of the in-place modes
    float* d_scratch = nullptr;
    // base pools of binary16 / bfloat16 values (PhiStorage): the float
    // pointers above then address 16-bit data; d_wide holds a binary32 copy
    // of the current pool for the diagnostics and read-outs
    int store = 0;
    float* d_wide = nullptr;
    size_t vbytes() const { return store ? 2 : 4; }

    void drop_graph() {
        if (graph_exec) cudaGraphExecDestroy(graph_exec);
        if (graph) cudaGraphDestroy(graph);
        graph_exec = nullptr;
        graph = nullptr;
    }

    ~pfb_sim3d() {
        drop_graph();
        if (bnd) (void)pfb::boundary3d_close(bnd, 0);  // unterminated: not a completed run
        if (stream) cudaStreamDestroy(stream);
        cudaFree(d_phi[0]);
        cudaFree(d_phi[1]);
        cudaFree(d_S[0]);
        cudaFree(d_S[1]);
        cudaFree(d_cells);
        cudaFree(d_accepted);
        cudaFree(d_flags);
        cudaFree(d_step);
        cudaFree(d_wall);
        cudaFree(d_wall_psi);
        cudaFree(d_centres);
        cudaFree(d_order);
        for (int b = 0; b < 2; ++b) {
            for (float* c : h_cube[b]) cudaFree(c);
            cudaFree(d_cube[b]);
        }
        cudaFree(d_prom_ids);
        cudaFree(d_requests);
        cudaFree(d_scratch);
        cudaFree(d_wide);
    }
    int prom_count() const { return (int)prom_ids.size(); }
};

namespace pfb {
namespace p3 {
int geometry_ok3(int B, const pfb_layout3d& L);
}
}  // namespace pfb

namespace {

// Channel wall diagnostics of each cell (reference src/pf3d/kernels.cu,
// k_measure_wall_diagnostics): FP64 sums over the brick's in-domain voxels
// of phi^2 psi_w^2(z) (wall overlap) and of phi^2 outside the slit. One CTA
// per cell; warp sums, then ascending warps.
constexpr int kWallThreads = 256;
// Brick of cell n: its own cube (edge = storage edge) when it has one, else
// its slot of the base pool.
__device__ __forceinline__ const float* cell_brick(const float* phi, float* const* cubes,
                                                  const pfb_cell3d* cells, int n, int B, int* E) {
    if (cubes && cubes[n]) {
        *E = (int)cells[n].storage_edge;
        return cubes[n];
    }
    *E = B;
    return phi + (size_t)n * B * B * B;
}

__global__ void __launch_bounds__(kWallThreads)
    k_wall_diag3d(const float* phi, float* const* cubes, pfb_cell3d* cells, int B0, int nz, int pad,
                  int H, const float* psi) {
    const int n = blockIdx.x;
    int B;
    const float* brick = cell_brick(phi, cubes, cells, n, B0, &B);
    const size_t words = (size_t)B * B * B, plane = (size_t)B * B;
    const int64_t oz = cells[n].origin_z;
    double overlap = 0.0, outside = 0.0;
    for (size_t q = threadIdx.x; q < words; q += kWallThreads) {
        const int64_t z = oz + (int64_t)(q / plane);
        if (z < 0 || z >= nz) continue;
        const double v = (double)brick[q];
        const double sq = v * v;
        overlap += sq * (double)psi[z];
        if (z < pad || z >= pad + H) outside += sq;
    }
    __shared__ double wo[kWallThreads / 32], wt[kWallThreads / 32];
    for (int d = 16; d; d >>= 1) {
        overlap += __shfl_down_sync(0xFFFFFFFFu, overlap, d);
        outside += __shfl_down_sync(0xFFFFFFFFu, outside, d);
    }
    if ((threadIdx.x & 31) == 0) {
        wo[threadIdx.x >> 5] = overlap;
        wt[threadIdx.x >> 5] = outside;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, b = 0.0;
        for (int w = 0; w < kWallThreads / 32; ++w) {
            a += wo[w];
            b += wt[w];
        }
        cells[n].wall_overlap = a;
        cells[n].outside_slit_volume = b;
    }
}

// Invariant check of each cell (reference src/pf3d/kernels.cu verify_one_cell):
// FP64 volume of the in-domain voxels, non-finite samples, and support
// voxels (|phi| > eps) on a brick face, outside the domain or on the slab's
// top plane. One CTA per cell.
struct Verify3 {
    double V;
    unsigned int nonfinite, edge;
};
__global__ void __launch_bounds__(kWallThreads)
    k_verify3d(const float* phi, float* const* cubes, const pfb_cell3d* cells, int B0, int nz,
               int periodic, int slab, Verify3* out) {
    const int n = blockIdx.x;
    int B;
    const float* brick = cell_brick(phi, cubes, cells, n, B0, &B);
    const size_t words = (size_t)B * B * B, plane = (size_t)B * B;
    const int64_t oz = cells[n].origin_z;
    double vol = 0.0;
    unsigned bad = 0, edge = 0;
    for (size_t q = threadIdx.x; q < words; q += kWallThreads) {
        const float v = brick[q];
        if (!isfinite(v)) {
            ++bad;
            continue;
        }
        const int z = (int)(q / plane);
        const int64_t wz = oz + z;
        const bool in = periodic || (wz >= 0 && wz < nz);
        const bool support = fabsf(v) > kSupportEps3;
        if (!in) {
            edge += support ? 1u : 0u;
            continue;
        }
        vol += (double)v * (double)v;
        if (support) {
            const int x = (int)(q % B), y = (int)((q / B) % B);
            edge += (x == 0 || x == B - 1 || y == 0 || y == B - 1 || z == 0 || z == B - 1 ||
                     (slab && wz == nz - 1))
                        ? 1u
                        : 0u;
        }
    }
    __shared__ double sv[kWallThreads / 32];
    __shared__ unsigned sb[kWallThreads / 32], se[kWallThreads / 32];
    for (int d = 16; d; d >>= 1) vol += __shfl_down_sync(0xFFFFFFFFu, vol, d);
    bad = __reduce_add_sync(0xFFFFFFFFu, bad);
    edge = __reduce_add_sync(0xFFFFFFFFu, edge);
    if ((threadIdx.x & 31) == 0) {
        sv[threadIdx.x >> 5] = vol;
        sb[threadIdx.x >> 5] = bad;
        se[threadIdx.x >> 5] = edge;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        Verify3 r{0.0, 0u, 0u};
        for (int w = 0; w < kWallThreads / 32; ++w) {
            r.V += sv[w];
            r.nonfinite += sb[w];
            r.edge += se[w];
        }
        out[n] = r;
    }
}

__global__ void k_max_u32(const uint32_t* a, size_t n, uint32_t* out) {
    uint32_t m = 0;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        m = max(m, a[i]);
    m = __reduce_max_sync(0xFFFFFFFFu, m);
    if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

double volume0(const pfb_params3d& p) {
    const double sphere = 4.0 * kPi * p.target_radius * p.target_radius * p.target_radius / 3.0;
    return substrate_slab(p.boundary_flags) ? 0.5 * sphere : sphere;
}

uint64_t polarity_stream(const pfb_params3d& p) { return p.polarity_seed ? p.polarity_seed : p.seed; }

constexpr long long kOrderRefresh = 4096;

// 21 bits of each coordinate interleaved (x lowest).
uint64_t morton3(uint32_t x, uint32_t y, uint32_t z) {
    auto spread = [](uint64_t v) {
        v &= 0x1FFFFFull;
        v = (v | (v << 32)) & 0x1F00000000FFFFull;
        v = (v | (v << 16)) & 0x1F0000FF0000FFull;
        v = (v | (v << 8)) & 0x100F00F00F00F00Full;
        v = (v | (v << 4)) & 0x10C30C30C30C30C3ull;
        v = (v | (v << 2)) & 0x1249249249249249ull;
        return v;
    };
    return spread(x) | (spread(y) << 1) | (spread(z) << 2);
}

// Visit order: Morton order of the (wrapped) brick centres, or the identity.
int refresh_order(pfb_sim3d* s) {
    std::vector<int> order((size_t)s->N);
    for (int i = 0; i < s->N; ++i) order[(size_t)i] = i;
    if (s->use_order) {
        std::vector<pfb_cell3d> c((size_t)s->N);
        PFB3_CU(cudaStreamSynchronize(s->stream), "sync");
        PFB3_CU(cudaMemcpy(c.data(), s->d_cells, c.size() * sizeof(pfb_cell3d), cudaMemcpyDeviceToHost),
                "read cells");
        const int h = s->B / 2;
        std::vector<uint64_t> key((size_t)s->N);
        for (int i = 0; i < s->N; ++i) {
            const pfb_cell3d& r = c[(size_t)i];
            const int x = wrap_origin(r.origin_x + h, s->L.nx);
            const int y = wrap_origin(r.origin_y + h, s->L.ny);
            const int64_t zz = r.origin_z + h;
            const int z = periodic_xyz(s->L.boundary_flags) ? wrap_origin(zz, s->L.nz)
                                                            : (int)std::max<int64_t>(0, zz);
            key[(size_t)i] = morton3((uint32_t)x, (uint32_t)y, (uint32_t)z);
        }
        std::stable_sort(order.begin(), order.end(),
                         [&](int a, int b) { return key[(size_t)a] < key[(size_t)b]; });
    }
    PFB3_CU(cudaStreamSynchronize(s->stream), "sync");
    PFB3_CU(cudaMemcpy(s->d_order, order.data(), order.size() * sizeof(int), cudaMemcpyHostToDevice),
            "upload order");
    s->order_step = s->steps_done;
    return PFB_OK;
}

int validate3(const pfb_params3d& p) {
    const uint32_t b = p.boundary_flags;
    if (periodic_xyz(b)) {
        if (p.Nx <= 0 || p.Nx != p.Ny || p.Nx != p.Nz)
            return set_error(PFB_E_ARG, "the periodic domain must be a positive cube");
    } else if (substrate_slab(b) || hard_wall_channel(b)) {
        if (p.Nx <= 0 || p.Ny != p.Nx || p.Nz <= 0)
            return set_error(PFB_E_ARG, "bounded-z geometry must have positive Nx=Ny and Nz");
    } else {
        return set_error(PFB_E_ARG, "unknown boundary flags");
    }
    if (hard_wall_channel(b)) {
        if (p.channel_height <= 0 || p.channel_padding <= 0 || !(p.wall_width > 0.0) ||
            !(p.wall_kappa > 0.0) || !(p.kappa > 0.0))
            return set_error(PFB_E_ARG, "channel wall parameters must be positive");
        if (p.channel_height + 2 * p.channel_padding != p.Nz)
            return set_error(PFB_E_ARG, "channel Nz must equal H + 2*padding");
    }
    if (p.num_cells <= 0) return set_error(PFB_E_ARG, "num_cells must be positive");
    if (p.phi_storage < 0 || p.phi_storage > 2) return set_error(PFB_E_ARG, "phi_storage must be 0, 1 or 2");
    if (!(p.dt > 0.0) || !(p.lambda > 0.0) || !(p.target_radius > 0.0) || !(p.xi > 0.0) ||
        !(p.tau > 0.0) || p.kappa < 0.0 || p.mu < 0.0 || p.v_A < 0.0 || !(p.gamma > 0.0))
        return set_error(PFB_E_ARG, "invalid model parameters");
    if (!(p.soft_fraction >= 0.0 && p.soft_fraction <= 1.0) ||
        (p.soft_fraction > 0.0 && !(p.gamma_soft > 0.0)))
        return set_error(PFB_E_ARG, "soft fraction must lie in [0, 1] with a positive gamma_soft");
    const double gmax = p.soft_fraction > 0.0 ? std::max(p.gamma, p.gamma_soft) : p.gamma;
    if (p.dt * gmax * (256.0 / 30.0) >= 1.0)
        return set_error(PFB_E_ARG, "explicit-Euler Laplacian stability bound is violated");
    return PFB_OK;
}

int upload_wall(pfb_sim3d* s) {
    const pfb_params3d& p = s->p;
    std::vector<float> w((size_t)p.Nz), psi((size_t)p.Nz);
    const float ratio = (float)(p.wall_kappa / p.kappa);
    const double k = 2.7386127875258306 / p.wall_width;
    const double lo = (double)p.channel_padding, hi = lo + p.channel_height;
    for (int z = 0; z < p.Nz; ++z) {
        const double c = (double)z + 0.5;
        const double fluid = 0.25 * (1.0 + std::tanh(k * (c - lo))) * (1.0 - std::tanh(k * (c - hi)));
        const double wall = 1.0 - fluid;
        psi[(size_t)z] = (float)(wall * wall);
        w[(size_t)z] = ratio * psi[(size_t)z];
    }
    PFB3_CU(cudaMalloc(&s->d_wall_psi, psi.size() * sizeof(float)), "cudaMalloc(wall psi)");
    PFB3_CU(cudaMemcpyAsync(s->d_wall_psi, psi.data(), psi.size() * sizeof(float),
                            cudaMemcpyHostToDevice, s->stream),
            "upload wall psi");
    PFB3_CU(cudaMalloc(&s->d_wall, w.size() * sizeof(float)), "cudaMalloc(wall)");
    PFB3_CU(cudaMemcpyAsync(s->d_wall, w.data(), w.size() * sizeof(float), cudaMemcpyHostToDevice,
                            s->stream),
            "upload wall field");
    return PFB_OK;
}

pfb_measure_args3d measure_args(pfb_sim3d* s, bool tumble, bool surface) {
    pfb_measure_args3d m{};
    m.phi = s->d_phi[s->cur_phi];
    m.S = s->d_S[s->cur_S];
    m.wall.values = s->d_wall;
    m.wall.planes = s->d_wall ? s->L.nz : 0;
    m.cells = s->d_cells;
    m.global_flags = s->d_flags;
    m.step = s->d_step;
    m.layout = s->L;
    m.N = s->N;
    m.B = s->B;
    m.shards = 1;
    m.polarity_stream = polarity_stream(s->p);
    const double aging = s->p.aging_time / s->p.dt + 0.5;
    m.aging_steps = (uint64_t)(aging > 0.0 ? aging : 0.0);
    m.p_tumble = -std::expm1(-s->p.dt / s->p.tau);
    m.motility_coeff = (float)(coeff_interaction(s->p.kappa, s->p.lambda) / s->p.xi);
    m.max_shift = kMaxShift3;
    m.support_margin = (int)kSafetyMargin;
    m.apply_tumble = tumble ? 1 : 0;
    m.compute_surface = surface ? 1 : 0;
    m.selection.ids = s->d_order;
    m.selection.count = s->N;
    return m;
}

pfb_update_args3d update_args(pfb_sim3d* s) {
    pfb_update_args3d u{};
    u.phi_in = s->d_phi[s->cur_phi];
    u.phi_out = s->mem_mode == 0 ? s->d_phi[1 - s->cur_phi] : nullptr;  // in place: none
    u.S_in = s->d_S[s->cur_S];
    u.S_out = s->mem_mode == 2 ? nullptr : s->d_S[1 - s->cur_S];       // compact: rebuilt
    u.wall.values = s->d_wall;
    u.wall.planes = s->d_wall ? s->L.nz : 0;
    u.cells = s->d_cells;
    u.global_flags = s->d_flags;
    u.layout = s->L;
    u.N = s->N;
    u.B = s->B;
    u.dt = (float)s->p.dt;
    u.V0 = s->V0;
    u.volume_scale = coeff_volume(s->p.mu, s->V0);
    u.bulk_scale = (float)coeff_bulk(s->p.lambda);
    u.interaction_coeff = (float)coeff_interaction(s->p.kappa, s->p.lambda);
    u.tile_pass = PFB3D_TILE_PASS_ALL;
    u.selection.ids = s->d_order;
    u.selection.count = s->N;
    return u;
}

bool full_step(const pfb_sim3d* s, long long step) {
    return s->p.full_moment_every > 0 && step % s->p.full_moment_every == 0;
}

// The current base pool as binary32 (a widened copy for 16-bit pools).
int wide_pool(pfb_sim3d* s, const float** out) {
    if (!s->store) {
        *out = s->d_phi[s->cur_phi];
        return PFB_OK;
    }
    const size_t n = (size_t)s->N * s->cell_words;
    if (!s->d_wide) PFB3_CU(cudaMalloc(&s->d_wide, n * sizeof(float)), "cudaMalloc(widened pool)");
    PFB3_RC(widen_pool(s->d_phi[s->cur_phi], s->d_wide, n, s->store, s->stream));
    *out = s->d_wide;
    return PFB_OK;
}

// Base slot n of pool b, in bytes of the storage type.
void* pool_slot(pfb_sim3d* s, int b, int n) {
    return static_cast<char*>(static_cast<void*>(s->d_phi[b])) + (size_t)n * s->cell_words * s->vbytes();
}

// The launches of one step on the current buffers (no host state changes).
int launch_step(pfb_sim3d* s, bool full) {
    PFB3_CU(cudaMemcpyAsync(s->d_accepted, s->d_cells, (size_t)s->N * sizeof(pfb_cell3d),
                            cudaMemcpyDeviceToDevice, s->stream),
            "snapshot accepted cells");
    const pfb_measure_args3d m = measure_args(s, true, full);
    const pfb_update_args3d u = update_args(s);
    const int np = s->prom_count();
    float* const* cur = s->d_cube[s->cur_cube];
    float* const* nxt = s->d_cube[1 - s->cur_cube];
    if (s->fused && np == 0 && s->mem_mode == 0 && s->store == 0) {
        PFB3_RC(clear3d_launch(s->d_S[1 - s->cur_S], &s->L, nullptr, s->stream));
        PFB3_RC(step3d_launch(&m, &u, s->stream));
    } else {
        // base bricks, then the promoted cubes; motion after every measurement
        PFB3_RC(measure3d_launch_pool(&m, s->store, s->stream));
        if (np) PFB3_RC(measure3d_promoted_launch(&m, cur, s->d_prom_ids, np, s->max_edge, s->stream));
        PFB3_RC(motion3d_launch(&m, s->stream));
        if (u.S_out) PFB3_RC(clear3d_launch(u.S_out, &s->L, nullptr, s->stream));
        if (s->mem_mode == 0)
            PFB3_RC(update3d_launch_pool(&u, s->store, s->d_step, s->p.seed, s->stream));
        else
            PFB3_RC(update3d_inplace_launch_pool(&u, s->d_scratch, s->slots, s->store, s->d_step, s->p.seed,
                                                 s->stream));
        if (np)
            PFB3_RC(update3d_promoted_launch(&u, cur, nxt, s->d_prom_ids, np, s->max_edge, s->stream));
    }
    PFB3_RC(repair3d_launch_pool(&u, s->store, s->stream));
    if (np) PFB3_RC(repair3d_promoted_launch(&u, cur, nxt, s->d_prom_ids, np, s->max_edge, s->stream));
    PFB3_RC(pfb3d_finalize_origins(s->d_cells, s->N, s->d_flags, s->stream));
    PFB3_RC(pfb3d_restore_cells_after_fatal(s->d_cells, s->d_accepted, s->N, s->d_flags,
                                            s->d_requests, s->stream));
    if (s->mem_mode == 2) {
        // compact: the single aggregate is rebuilt from the new fields
        // (reference Sim3D::finish_step, src/pf3d/sim.cu:1636-1641)
        PFB3_RC(clear3d_launch(s->d_S[0], &s->L, nullptr, s->stream));
        pfb_scatter_args3d sa{};
        sa.phi = s->d_phi[0];
        sa.cells = s->d_cells;
        sa.S = s->d_S[0];
        sa.global_flags = s->d_flags;
        sa.layout = s->L;
        sa.N = s->N;
        sa.B = s->B;
        PFB3_RC(scatter3d_launch_pool(&sa, s->store, s->stream));
        if (np) PFB3_RC(scatter3d_promoted_launch(&sa, nxt, s->d_prom_ids, np, s->max_edge, 0, s->stream));
    }
    PFB3_RC(pfb3d_advance_step(s->d_step, s->d_flags, s->stream));
    return PFB_OK;
}

void flip(pfb_sim3d* s) {
    if (s->mem_mode == 0) s->cur_phi = 1 - s->cur_phi;
    if (s->mem_mode != 2) s->cur_S = 1 - s->cur_S;
    s->cur_cube = 1 - s->cur_cube;
}

int one_step(pfb_sim3d* s) {
    PFB3_RC(launch_step(s, full_step(s, s->steps_done)));
    flip(s);
    ++s->steps_done;
    return PFB_OK;
}

// The current aggregate rebuilt from the current fields (reference
// Sim3D::reconstruct_current_S).
int reconstruct_S(pfb_sim3d* s) {
    PFB3_RC(clear3d_launch(s->d_S[s->cur_S], &s->L, nullptr, s->stream));
    pfb_scatter_args3d sa{};
    sa.phi = s->d_phi[s->cur_phi];
    sa.cells = s->d_cells;
    sa.S = s->d_S[s->cur_S];
    sa.global_flags = s->d_flags;
    sa.layout = s->L;
    sa.N = s->N;
    sa.B = s->B;
    PFB3_RC(scatter3d_launch_pool(&sa, s->store, s->stream));
    if (s->prom_count())
        PFB3_RC(scatter3d_promoted_launch(&sa, s->d_cube[s->cur_cube], s->d_prom_ids, s->prom_count(),
                                          s->max_edge, 0, s->stream));
    return PFB_OK;
}

// Measurement of every cell on the current field (no tumble); the motion
// only when asked (reference Sim3D::refresh_measurements).
int refresh(pfb_sim3d* s, bool surface, bool motion) {
    const pfb_measure_args3d m = measure_args(s, false, surface);
    PFB3_RC(measure3d_launch_pool(&m, s->store, s->stream));
    if (s->prom_count())
        PFB3_RC(measure3d_promoted_launch(&m, s->d_cube[s->cur_cube], s->d_prom_ids, s->prom_count(),
                                          s->max_edge, s->stream));
    if (motion) PFB3_RC(motion3d_launch(&m, s->stream));
    return PFB_OK;
}

int edge_of(const pfb_sim3d* s, const pfb_cell3d& c) {
    return c.storage_edge > (uint32_t)s->B ? (int)c.storage_edge : s->B;
}

// A cell record moved into a centred cube of edge En (reference
// adaptive_storage.cu translate_state): the world field stays in place.
bool translate_record(pfb_cell3d* c, int Eo, int En) {
    const int off = (En - Eo) / 2;
    int64_t* o[3] = {&c->origin_x, &c->origin_y, &c->origin_z};
    for (int64_t* v : o) {
        if ((off > 0 && *v < INT64_MIN + off) || (off < 0 && *v > INT64_MAX + off)) return false;
        *v -= off;
    }
    c->Cx += (double)off * c->V;
    c->Cy += (double)off * c->V;
    c->Cz += (double)off * c->V;
    if (!std::isfinite(c->Cx) || !std::isfinite(c->Cy) || !std::isfinite(c->Cz)) return false;
    if (c->bb_hi_x >= c->bb_lo_x) {
        c->bb_lo_x += off; c->bb_hi_x += off;
        c->bb_lo_y += off; c->bb_hi_y += off;
        c->bb_lo_z += off; c->bb_hi_z += off;
    }
    c->pending_shift_x = c->pending_shift_y = c->pending_shift_z = 0;
    c->storage_edge = (uint32_t)En;
    c->flags &= ~((1u << PFB3D_FLAG_SUPPORT_EXHAUSTED) | (1u << PFB3D_FLAG_SUPPORT_EDGE));
    return true;
}

int upload_tables(pfb_sim3d* s) {
    for (int b = 0; b < 2; ++b)
        PFB3_CU(cudaMemcpy(s->d_cube[b], s->h_cube[b].data(), (size_t)s->N * sizeof(float*),
                           cudaMemcpyHostToDevice),
                "upload cube table");
    if (!s->prom_ids.empty())
        PFB3_CU(cudaMemcpy(s->d_prom_ids, s->prom_ids.data(), s->prom_ids.size() * sizeof(int),
                           cudaMemcpyHostToDevice),
                "upload promoted ids");
    return PFB_OK;
}

// Move the requested cells (id, new edge) into centred cubes of the new edge
// (a new edge equal to B returns the cell to its base slot), transactionally:
// every new cube is allocated and filled before any table changes (reference
// Sim3D::resize_cells). `cells` holds the current records on entry and the
// installed ones on success.
int resize_cells(pfb_sim3d* s, const std::vector<std::pair<int, int>>& req,
                 std::vector<pfb_cell3d>* cells) {
    PFB3_CU(cudaStreamSynchronize(s->stream), "sync");
    std::vector<pfb_cell3d> next = *cells;
    struct Move { int id, Eo, En; float* cube[2]; };
    std::vector<Move> moves;
    auto release = [&]() {
        for (Move& m : moves)
            for (float* c : m.cube) cudaFree(c);
    };
    for (const auto& r : req) {
        const int n = r.first, En = r.second;
        const int Eo = edge_of(s, (*cells)[(size_t)n]);
        if (n < 0 || n >= s->N || En < s->B || En > s->max_edge || En % kBrickAlign != 0 || En == Eo ||
            !translate_record(&next[(size_t)n], Eo, En)) {
            release();
            return set_error(PFB_E_STATE, "resize of cell %d from %d to %d refused", n, Eo, En);
        }
        Move m{n, Eo, En, {nullptr, nullptr}};
        if (En > s->B)
            for (float*& c : m.cube)
                if (cudaMalloc(&c, (size_t)En * En * En * sizeof(float)) != cudaSuccess) {
                    moves.push_back(m);
                    release();
                    return set_error(PFB_E_NOMEM, "no device memory for a %d^3 cube of cell %d", En, n);
                }
        moves.push_back(m);
    }
    const size_t bw = (size_t)s->B * s->B * s->B;
    const float* wide = nullptr;
    float* brick = nullptr;  // a binary32 base brick on its way into a 16-bit pool
    int rc0 = wide_pool(s, &wide);
    if (!rc0 && s->store && cudaMalloc(&brick, bw * sizeof(float)) != cudaSuccess)
        rc0 = set_error(PFB_E_NOMEM, "no device memory for a staging brick");
    for (Move& m : moves) {
        const float* src = m.Eo > s->B ? s->h_cube[s->cur_cube][(size_t)m.id] : wide + (size_t)m.id * bw;
        for (int b = 0; b < 2 && !rc0; ++b) {
            if (m.En == s->B && !s->d_phi[b]) continue;  // one pool in place
            if (m.En > s->B) {
                rc0 = copy_centred3d_launch(src, m.Eo, m.cube[b], m.En, s->stream);
            } else if (!s->store) {
                rc0 = copy_centred3d_launch(src, m.Eo, s->d_phi[b] + (size_t)m.id * bw, m.En, s->stream);
            } else {
                rc0 = copy_centred3d_launch(src, m.Eo, brick, m.En, s->stream);
                if (!rc0) rc0 = narrow_pool(brick, pool_slot(s, b, m.id), bw, s->store, s->stream);
            }
        }
    }
    if (rc0) {
        cudaStreamSynchronize(s->stream);
        cudaFree(brick);
        release();
        return rc0;
    }
    if (cudaStreamSynchronize(s->stream) != cudaSuccess) {
        cudaFree(brick);
        release();
        return set_error(PFB_E_CUDA, "cube copies failed");
    }
    cudaFree(brick);
    // install: tables, id list, records; then free the replaced cubes
    for (Move& m : moves)
        for (int b = 0; b < 2; ++b) {
            float* old = s->h_cube[b][(size_t)m.id];
            s->h_cube[b][(size_t)m.id] = m.cube[b];
            m.cube[b] = old;
        }
    s->prom_ids.clear();
    for (int n = 0; n < s->N; ++n)
        if (next[(size_t)n].storage_edge > (uint32_t)s->B) s->prom_ids.push_back(n);
    PFB3_RC(upload_tables(s));
    PFB3_CU(cudaMemcpy(s->d_cells, next.data(), next.size() * sizeof(pfb_cell3d), cudaMemcpyHostToDevice),
            "install resized records");
    s->prom_edge = 0;
    for (int n : s->prom_ids) s->prom_edge = std::max(s->prom_edge, (int)next[(size_t)n].storage_edge);
    release();  // the replaced cubes
    cells->swap(next);
    s->drop_graph();  // launch shapes changed
    return PFB_OK;
}

int read_flags(pfb_sim3d* s, uint32_t* f) {
    PFB3_CU(cudaStreamSynchronize(s->stream), "sync");
    PFB3_CU(cudaMemcpy(f, s->d_flags, PFB3D_FLAG_COUNT * sizeof(uint32_t), cudaMemcpyDeviceToHost),
            "read flags");
    return PFB_OK;
}

bool fatal_in(const uint32_t* f) {
    for (int i = 0; i < PFB3D_FLAG_COUNT; ++i)
        if (((PFB3D_FATAL_MASK >> i) & 1u) && f[i]) return true;
    return false;
}

// Support exhaustion as the only fatal flag: grow every requesting cell to the
// next tier, rebuild the aggregate, remeasure without motion and check again
// (reference Sim3D::recover_support_exhaustion). *ok false: not recoverable
// (the state is left as the rolled-back step left it).
int recover_support(pfb_sim3d* s, const uint32_t* flags, bool* ok) {
    *ok = false;
    if (!flags[PFB3D_FLAG_SUPPORT_EXHAUSTED]) return PFB_OK;
    for (int f = 0; f < PFB3D_FLAG_COUNT; ++f)
        if (f != PFB3D_FLAG_SUPPORT_EXHAUSTED && ((PFB3D_FATAL_MASK >> f) & 1u) && flags[f]) return PFB_OK;
    std::vector<pfb_cell3d> cells((size_t)s->N);
    std::vector<uint32_t> requests((size_t)s->N);
    PFB3_CU(cudaMemcpy(cells.data(), s->d_cells, cells.size() * sizeof(pfb_cell3d), cudaMemcpyDeviceToHost),
            "read cells");
    PFB3_CU(cudaMemcpy(requests.data(), s->d_requests, requests.size() * sizeof(uint32_t),
                       cudaMemcpyDeviceToHost),
            "read support requests");
    std::vector<std::pair<int, int>> req;
    for (int n = 0; n < s->N; ++n) {
        const pfb_cell3d& c = cells[(size_t)n];
        if (!requests[(size_t)n] && !(c.flags & (1u << PFB3D_FLAG_SUPPORT_EXHAUSTED))) continue;
        const int next = next_brick_edge3(edge_of(s, c), s->max_edge);
        if (next == 0 || next > kMaxPromotedEdge) return PFB_OK;  // no larger cube fits the domain
        req.emplace_back(n, next);
    }
    if (req.empty()) return PFB_OK;
    PFB3_RC(resize_cells(s, req, &cells));
    PFB3_CU(cudaMemsetAsync(s->d_flags + PFB3D_FLAG_SUPPORT_EXHAUSTED, 0, sizeof(uint32_t), s->stream),
            "clear flag");
    PFB3_CU(cudaMemsetAsync(s->d_flags + PFB3D_FLAG_SUPPORT_EDGE, 0, sizeof(uint32_t), s->stream),
            "clear flag");
    PFB3_CU(cudaMemsetAsync(s->d_requests, 0, (size_t)s->N * sizeof(uint32_t), s->stream), "clear requests");
    PFB3_RC(reconstruct_S(s));
    PFB3_RC(refresh(s, false, false));
    ++s->recoveries;
    uint32_t after[PFB3D_FLAG_COUNT];
    PFB3_RC(read_flags(s, after));
    if (after[PFB3D_FLAG_SUPPORT_EXHAUSTED]) return recover_support(s, after, ok);
    *ok = !fatal_in(after);
    return PFB_OK;
}

// Every kBrickCompactEvery accepted steps: crop promoted cubes whose support
// leaves enough exactly-zero shell (reference Sim3D::compact_promoted_fields).
int compact_cubes(pfb_sim3d* s) {
    if (s->prom_ids.empty()) return PFB_OK;
    PFB3_RC(refresh(s, false, false));  // support boxes of the accepted field
    std::vector<pfb_cell3d> cells((size_t)s->N);
    PFB3_CU(cudaStreamSynchronize(s->stream), "sync");
    PFB3_CU(cudaMemcpy(cells.data(), s->d_cells, cells.size() * sizeof(pfb_cell3d), cudaMemcpyDeviceToHost),
            "read cells");
    std::vector<int> cand((size_t)s->N, 0);
    bool any = false;
    for (int n : s->prom_ids) {
        const pfb_cell3d& c = cells[(size_t)n];
        const int lo[3] = {c.bb_lo_x, c.bb_lo_y, c.bb_lo_z}, hi[3] = {c.bb_hi_x, c.bb_hi_y, c.bb_hi_z};
        const int E = edge_of(s, c);
        const int smaller = shrink_brick_edge3(E, s->B, lo, hi);
        if (smaller < E) {
            cand[(size_t)n] = smaller;
            any = true;
        }
    }
    if (!any) return PFB_OK;
    int* d_cand = nullptr;
    uint32_t* d_rej = nullptr;
    std::vector<uint32_t> rej((size_t)s->N, 0u);
    int rc = PFB_OK;
    if (cudaMalloc(&d_cand, cand.size() * sizeof(int)) != cudaSuccess ||
        cudaMalloc(&d_rej, rej.size() * sizeof(uint32_t)) != cudaSuccess ||
        cudaMemcpy(d_cand, cand.data(), cand.size() * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemset(d_rej, 0, rej.size() * sizeof(uint32_t)) != cudaSuccess)
        rc = set_error(PFB_E_CUDA, "crop check buffers");
    if (!rc) rc = check_crops3d_launch(s->d_cube[s->cur_cube], s->d_cells, d_cand, d_rej, s->N, s->B, s->stream);
    if (!rc && (cudaStreamSynchronize(s->stream) != cudaSuccess ||
                cudaMemcpy(rej.data(), d_rej, rej.size() * sizeof(uint32_t), cudaMemcpyDeviceToHost) !=
                    cudaSuccess))
        rc = set_error(PFB_E_CUDA, "crop check");
    cudaFree(d_cand);
    cudaFree(d_rej);
    if (rc) return rc;
    std::vector<std::pair<int, int>> req;
    for (int n : s->prom_ids)
        if (cand[(size_t)n] && !rej[(size_t)n]) req.emplace_back(n, cand[(size_t)n]);
    if (req.empty()) return PFB_OK;
    PFB3_RC(resize_cells(s, req, &cells));
    PFB3_RC(reconstruct_S(s));
    PFB3_RC(refresh(s, false, false));
    return PFB_OK;
}

// Capture two steps without a surface pass, from buffer parity 0 (every
// double buffer back on the same side after them).
int build_graph(pfb_sim3d* s) {
    s->drop_graph();
    PFB3_CU(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal), "begin capture");
    int rc = launch_step(s, false);
    flip(s);
    if (rc == PFB_OK) rc = launch_step(s, false);
    flip(s);
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(s->stream, &g);
    if (rc != PFB_OK) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    PFB3_CU(e, "end capture");
    s->graph = g;
    PFB3_CU(cudaGraphInstantiateWithFlags(&s->graph_exec, s->graph, 0), "graph instantiate");
    return PFB_OK;
}

// Run `steps` step attempts (graph pairs where possible).
int attempt_steps(pfb_sim3d* s, long long steps) {
    while (steps > 0) {
        if (s->steps_done - s->order_step >= kOrderRefresh) PFB3_RC(refresh_order(s));
        const bool pair = s->use_graph && s->cur_cube == 0 && steps >= 2 &&
                          !full_step(s, s->steps_done) && !full_step(s, s->steps_done + 1);
        if (pair) {
            if (!s->graph_exec) PFB3_RC(build_graph(s));
            PFB3_CU(cudaGraphLaunch(s->graph_exec, s->stream), "graph launch");
            s->steps_done += 2;
            steps -= 2;
        } else {
            PFB3_RC(one_step(s));
            --steps;
        }
    }
    return PFB_OK;
}

// Advance by `steps` accepted steps. A step that exhausts a cell's support is
// rolled back; at the next synchronisation the cell's brick grows to the next
// tier and the rolled-back steps are retried. Stops early, leaving the flags
// for the caller, at any other fatal flag. Promoted cubes are compacted at
// every multiple of kBrickCompactEvery accepted steps.
int advance_impl(pfb_sim3d* s, long long steps) {
    const long long target = s->accepted + steps;
    while (s->accepted < target) {
        // synchronisations land on the compaction multiples
        const long long chunk = std::min(target, s->next_compact) - s->accepted;
        PFB3_RC(attempt_steps(s, chunk));
        uint32_t f[PFB3D_FLAG_COUNT];
        PFB3_RC(read_flags(s, f));
        uint64_t acc = 0;
        PFB3_CU(cudaMemcpy(&acc, s->d_step, sizeof(acc), cudaMemcpyDeviceToHost), "read step");
        s->accepted = (long long)acc;
        s->steps_done = s->accepted;
        if (fatal_in(f)) {
            bool ok = false;
            PFB3_RC(recover_support(s, f, &ok));
            if (!ok) return PFB_OK;
            continue;
        }
        if (s->accepted >= s->next_compact) {
            PFB3_RC(compact_cubes(s));
            s->next_compact = (s->accepted / kBrickCompactEvery + 1) * kBrickCompactEvery;
        }
    }
    return PFB_OK;
}

// Storage mode and scratch bricks (reference Sim3D::allocate storage
// selection, src/pf3d/sim.cu:440-560): mem_mode -1 (auto) takes throughput
// when two pools and two aggregates fit in 90 % of the free device memory,
// else balanced when one pool, two aggregates and a scratch brick per
// resident update cluster fit, else compact. slots 0: 2 per SM, at most N.
int choose_storage(pfb_sim3d* s) {
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int want = s->slots > 0 ? s->slots : std::min(s->N, 2 * sms);
    if (s->mode_request < -1 || s->mode_request > 2)
        return set_error(PFB_E_ARG, "unknown storage mode %d", s->mode_request);
    if (s->slots < 0 || s->slots > s->N) return set_error(PFB_E_ARG, "scratch slots must be 0..N");
    int mode = s->mode_request;
    if (mode < 0) {
        size_t free_b = 0, total_b = 0;
        if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) free_b = (size_t)-1;
        const double budget = 0.9 * (double)free_b;
        const double vb = (double)s->vbytes();
        const double pool = (double)s->N * (double)s->cell_words * vb, agg = (double)s->s_words * 4.0;
        const double brick = (double)s->cell_words * vb;
        mode = 2 * pool + 2 * agg <= budget ? 0 : pool + 2 * agg + want * brick <= budget ? 1 : 2;
    }
    s->mem_mode = mode;
    s->slots = mode == 0 ? 0 : want;
    return PFB_OK;
}

// Buffers, layout and wall field of a system with parameters *pp.
int alloc_impl(pfb_sim3d* s, const pfb_params3d* pp, int device) {
    s->p = *pp;
    const pfb_params3d& p = s->p;
    PFB3_RC(validate3(p));
    s->device = device;
    PFB3_CU(cudaSetDevice(device), "cudaSetDevice");
    s->B = p.B > 0 ? p.B : pfb3d_automatic_brick_edge(p.target_radius, p.lambda);
    if (s->B <= 0 || s->B % kBrickAlign != 0)
        return set_error(PFB_E_CONFIG, "brick edge must be a positive multiple of 8");
    s->N = p.num_cells;
    s->L.nx = p.Nx;
    s->L.ny = p.Ny;
    s->L.nz = p.Nz;
    s->L.pitch_x = (p.Nx + 31) / 32 * 32;
    s->L.boundary_flags = p.boundary_flags;
    if (!geometry_ok3(s->B, s->L)) return set_error(PFB_E_ARG, "the brick must fit inside the domain");
    s->V0 = volume0(p);
    s->store = p.phi_storage;
    s->fused = 0;  // the separate launches measure faster (both are issue-bound)
    s->s_words = (size_t)s->L.pitch_x * s->L.ny * s->L.nz;
    s->cell_words = (size_t)s->B * s->B * s->B;
    PFB3_CU(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking), "stream");
    PFB3_RC(choose_storage(s));
    for (int i = 0; i < 2; ++i) {
        if (i == 0 || s->mem_mode == 0)
            PFB3_CU(cudaMalloc(&s->d_phi[i], (size_t)s->N * s->cell_words * s->vbytes()), "cudaMalloc(phi)");
        if (i == 0 || s->mem_mode != 2)
            PFB3_CU(cudaMalloc(&s->d_S[i], s->s_words * sizeof(uint32_t)), "cudaMalloc(S)");
    }
    if (s->mem_mode != 0)
        PFB3_CU(cudaMalloc(&s->d_scratch, (size_t)s->slots * s->cell_words * s->vbytes()),
                "cudaMalloc(scratch bricks)");
    PFB3_CU(cudaMalloc(&s->d_cells, (size_t)s->N * sizeof(pfb_cell3d)), "cudaMalloc(cells)");
    PFB3_CU(cudaMalloc(&s->d_accepted, (size_t)s->N * sizeof(pfb_cell3d)), "cudaMalloc(cells)");
    PFB3_CU(cudaMalloc(&s->d_flags, PFB3D_FLAG_COUNT * sizeof(uint32_t)), "cudaMalloc(flags)");
    PFB3_CU(cudaMalloc(&s->d_step, sizeof(uint64_t)), "cudaMalloc(step)");
    PFB3_CU(cudaMalloc(&s->d_centres, (size_t)s->N * sizeof(pfb_vec3)), "cudaMalloc(centres)");
    PFB3_CU(cudaMalloc(&s->d_order, (size_t)s->N * sizeof(int)), "cudaMalloc(order)");
    {
        std::vector<int> id((size_t)s->N);
        for (int i = 0; i < s->N; ++i) id[(size_t)i] = i;
        PFB3_CU(cudaMemcpy(s->d_order, id.data(), id.size() * sizeof(int), cudaMemcpyHostToDevice),
                "upload order");
    }
    PFB3_CU(cudaMemsetAsync(s->d_flags, 0, PFB3D_FLAG_COUNT * sizeof(uint32_t), s->stream), "memset");
    PFB3_CU(cudaMemsetAsync(s->d_step, 0, sizeof(uint64_t), s->stream), "memset");
    // adaptive bricks: the largest cube that fits the domain (reference
    // src/pf3d/sim.cu:291-293), empty tables, no requests
    const int dom = hard_wall_channel(p.boundary_flags) ? std::min(p.Nx, p.Ny)
                                                        : std::min(std::min(p.Nx, p.Ny), p.Nz);
    s->max_edge = std::min((dom - 1) / kBrickAlign * kBrickAlign, kMaxPromotedEdge);
    for (int b = 0; b < 2; ++b) {
        s->h_cube[b].assign((size_t)s->N, nullptr);
        PFB3_CU(cudaMalloc(&s->d_cube[b], (size_t)s->N * sizeof(float*)), "cudaMalloc(cube table)");
        PFB3_CU(cudaMemsetAsync(s->d_cube[b], 0, (size_t)s->N * sizeof(float*), s->stream), "memset");
    }
    PFB3_CU(cudaMalloc(&s->d_prom_ids, (size_t)s->N * sizeof(int)), "cudaMalloc(promoted ids)");
    PFB3_CU(cudaMalloc(&s->d_requests, (size_t)s->N * sizeof(uint32_t)), "cudaMalloc(requests)");
    PFB3_CU(cudaMemsetAsync(s->d_requests, 0, (size_t)s->N * sizeof(uint32_t), s->stream), "memset");
    if (hard_wall_channel(p.boundary_flags)) PFB3_RC(upload_wall(s));
    return PFB_OK;
}

void set_accepted(pfb_sim3d* s, long long step) {
    s->accepted = step;
    s->steps_done = step;
    s->next_compact = (step / kBrickCompactEvery + 1) * kBrickCompactEvery;
}

// The measurement that follows a fresh seeding or a restore (reference
// Sim3D::refresh_measurements(false, true) after reconstruct_current_S,
// src/pf3d/sim.cu:877, 1175): aggregate from the current bricks, then
// moments, surface, recentring plan and velocities without a tumble.
int remeasure_impl(pfb_sim3d* s) {
    PFB3_RC(reconstruct_S(s));
    return refresh(s, true, true);
}

int create_impl(pfb_sim3d* s, const pfb_params3d* pp, const pfb_vec3* centres, int device) {
    PFB3_RC(alloc_impl(s, pp, device));
    const pfb_params3d& p = s->p;

    // per-cell records (reference src/pf3d/sim.cu:1100-1130)
    std::vector<uint8_t> soft((size_t)s->N, 0);
    if (p.soft_fraction > 0.0) PFB3_RC(pfb3d_soft_membership(s->N, p.soft_fraction, p.seed, soft.data()));
    std::vector<pfb_cell3d> cells((size_t)s->N);
    std::vector<pfb_vec3> ctr((size_t)s->N);
    const bool slab = substrate_slab(p.boundary_flags);
    for (int i = 0; i < s->N; ++i) {
        pfb_cell3d c;
        std::memset(&c, 0, sizeof(c));
        c.global_id = i;
        c.gamma = (float)(soft[(size_t)i] ? p.gamma_soft : p.gamma);
        c.v_A = (float)initial_speed3(i, p.seed, p.v_A, p.v_A_sigma);
        c.R_tgt = (float)p.target_radius;
        const Dir3 d = initial_polarity3(i, polarity_stream(p), slab);
        c.polarity_x = (float)d.x;
        c.polarity_y = (float)d.y;
        c.polarity_z = (float)d.z;
        cells[(size_t)i] = c;
        pfb_vec3 v = centres[i];
        // channel centres are given in slit coordinates; stored z adds the
        // padding minus half a plane (reference src/pf3d/sim.cu:1121-1124)
        if (hard_wall_channel(p.boundary_flags))
            v.z = (double)((float)v.z + (float)p.channel_padding - 0.5f);
        ctr[(size_t)i] = v;
    }
    PFB3_CU(cudaMemcpyAsync(s->d_cells, cells.data(), cells.size() * sizeof(pfb_cell3d),
                            cudaMemcpyHostToDevice, s->stream),
            "upload cells");
    PFB3_CU(cudaMemcpyAsync(s->d_centres, ctr.data(), ctr.size() * sizeof(pfb_vec3),
                            cudaMemcpyHostToDevice, s->stream),
            "upload centres");
    double seed = 0.0;
    PFB3_RC(pfb3d_calibrate_seed_radius(p.target_radius, p.lambda, s->B, &seed, nullptr));
    pfb_init_args3d ia{};
    float* seeded = nullptr;  // 16-bit pools: seeded in binary32, then rounded to nearest
    if (s->store) {
        PFB3_CU(cudaMalloc(&seeded, (size_t)s->N * s->cell_words * sizeof(float)), "cudaMalloc(seeding)");
        if (s->d_phi[1])
            PFB3_CU(cudaMemsetAsync(s->d_phi[1], 0, (size_t)s->N * s->cell_words * s->vbytes(), s->stream),
                    "clear pool");
    }
    ia.phi_even = s->store ? seeded : s->d_phi[0];
    ia.phi_odd = s->store ? nullptr : s->d_phi[1];
    ia.cells = s->d_cells;
    ia.centres = s->d_centres;
    ia.N = s->N;
    ia.B = s->B;
    ia.layout = s->L;
    ia.lambda = (float)p.lambda;
    ia.seed_radius = (float)seed;
    int rc = init3d_launch(&ia, s->stream);
    if (!rc && s->store) rc = narrow_pool(seeded, s->d_phi[0], (size_t)s->N * s->cell_words, s->store, s->stream);
    if (seeded) {
        cudaStreamSynchronize(s->stream);
        cudaFree(seeded);
    }
    PFB3_RC(rc);
    PFB3_RC(remeasure_impl(s));
    PFB3_CU(cudaStreamSynchronize(s->stream), "fresh initialisation");
    set_accepted(s, 0);
    return refresh_order(s);
}

// Restore (reference Sim3D::init_checkpoint and install_checkpoint_promotions,
// src/pf3d/sim.cu:794-885, adaptive_storage.cu:264-310): cell records and
// fields of step `step` into the current buffers, the step counter, then the
// aggregate and one measurement. `phi` packs each cell's field in cell order:
// B^3 values for a base cell, E^3 for a cell whose storage edge E exceeds B.
int restore_impl(pfb_sim3d* s, const pfb_params3d* pp, const pfb_cell3d* cells_in, const float* phi,
                 long long step, int device) {
    if (!cells_in || !phi || step < 0) return set_error(PFB_E_ARG, "restore: bad argument");
    PFB3_RC(alloc_impl(s, pp, device));
    std::vector<pfb_cell3d> cells(cells_in, cells_in + s->N);
    for (int i = 0; i < s->N; ++i) {
        pfb_cell3d& c = cells[(size_t)i];
        if (c.storage_edge == (uint32_t)s->B) c.storage_edge = 0;  // a base record
        const bool ok = c.global_id == i &&
                        (c.storage_edge == 0 ||
                         (c.storage_edge > (uint32_t)s->B && (int)c.storage_edge <= s->max_edge &&
                          c.storage_edge % kBrickAlign == 0));
        if (!ok) return set_error(PFB_E_ARG, "restore: cell %d has an invalid id or storage edge", i);
    }
    const size_t bw = s->cell_words;
    size_t off = 0;
    // 16-bit pools: the base bricks go through a binary32 copy, rounded to nearest
    float* staged = s->d_phi[0];
    if (s->store) PFB3_CU(cudaMalloc(&staged, (size_t)s->N * bw * sizeof(float)), "cudaMalloc(staging)");
    for (int i = 0; i < s->N; ++i) {
        const int E = edge_of(s, cells[(size_t)i]);
        const size_t words = (size_t)E * E * E;
        if (E == s->B) {
            PFB3_CU(cudaMemcpy(staged + (size_t)i * bw, phi + off, words * sizeof(float),
                               cudaMemcpyHostToDevice),
                    "upload brick");
        } else {
            for (int b = 0; b < 2; ++b) {
                PFB3_CU(cudaMalloc(&s->h_cube[b][(size_t)i], words * sizeof(float)), "cudaMalloc(cube)");
                PFB3_CU(cudaMemcpy(s->h_cube[b][(size_t)i], phi + off, words * sizeof(float),
                                   cudaMemcpyHostToDevice),
                        "upload cube");
            }
            s->prom_ids.push_back(i);
            s->prom_edge = std::max(s->prom_edge, E);
        }
        off += words;
    }
    if (s->store) {
        const int rc = narrow_pool(staged, s->d_phi[0], (size_t)s->N * bw, s->store, s->stream);
        cudaStreamSynchronize(s->stream);
        cudaFree(staged);
        PFB3_RC(rc);
    }
    PFB3_RC(upload_tables(s));
    PFB3_CU(cudaMemcpyAsync(s->d_cells, cells.data(), (size_t)s->N * sizeof(pfb_cell3d), cudaMemcpyHostToDevice,
                            s->stream), "upload cells");
    if (s->d_phi[1])
        PFB3_CU(cudaMemsetAsync(s->d_phi[1], 0, (size_t)s->N * s->cell_words * s->vbytes(), s->stream),
                "clear phi");
    const uint64_t st = (uint64_t)step;
    PFB3_CU(cudaMemcpyAsync(s->d_step, &st, sizeof(st), cudaMemcpyHostToDevice, s->stream), "step");
    set_accepted(s, step);
    s->cur_phi = 0;
    s->cur_S = 0;
    s->cur_cube = 0;
    PFB3_RC(remeasure_impl(s));
    PFB3_CU(cudaStreamSynchronize(s->stream), "restore");
    return refresh_order(s);
}

// Values of the packed field of the current state (each cell's own edge).
size_t packed_words(const pfb_sim3d* s, const std::vector<pfb_cell3d>& cells) {
    size_t w = 0;
    for (const pfb_cell3d& c : cells) {
        const size_t E = (size_t)edge_of(s, c);
        w += E * E * E;
    }
    return w;
}

}  // namespace

extern "C" {

pfb_sim3d* pfb_sim3d_create_ex(const pfb_params3d* p, const pfb_vec3* centres, int device, int memory_mode,
                               int scratch_slots) {
    clear_error();
    if (!p || !centres) {
        set_error(PFB_E_ARG, "null params or centres");
        return nullptr;
    }
    pfb_sim3d* s = new (std::nothrow) pfb_sim3d();
    if (!s) {
        set_error(PFB_E_NOMEM, "host allocation failed");
        return nullptr;
    }
    s->mode_request = memory_mode;
    s->slots = scratch_slots;
    if (create_impl(s, p, centres, device) != PFB_OK) {
        delete s;
        return nullptr;
    }
    return s;
}

pfb_sim3d* pfb_sim3d_create(const pfb_params3d* p, const pfb_vec3* centres, int device) {
    return pfb_sim3d_create_ex(p, centres, device, PFB3D_MEMORY_AUTO, 0);
}

pfb_sim3d* pfb_sim3d_create_from_state_ex(const pfb_params3d* p, const pfb_cell3d* cells, const float* phi,
                                          long long step, int device, int memory_mode, int scratch_slots) {
    clear_error();
    if (!p || !cells || !phi) {
        set_error(PFB_E_ARG, "null params, cells or phi");
        return nullptr;
    }
    pfb_sim3d* s = new (std::nothrow) pfb_sim3d();
    if (!s) {
        set_error(PFB_E_NOMEM, "host allocation failed");
        return nullptr;
    }
    s->mode_request = memory_mode;
    s->slots = scratch_slots;
    if (restore_impl(s, p, cells, phi, step, device) != PFB_OK) {
        delete s;
        return nullptr;
    }
    return s;
}

pfb_sim3d* pfb_sim3d_create_from_state(const pfb_params3d* p, const pfb_cell3d* cells,
                                       const float* phi, long long step, int device) {
    return pfb_sim3d_create_from_state_ex(p, cells, phi, step, device, PFB3D_MEMORY_AUTO, 0);
}

int pfb_sim3d_memory_mode(const pfb_sim3d* s) { return s ? s->mem_mode : -1; }

int pfb_sim3d_scratch_slots(const pfb_sim3d* s) { return s ? s->slots : -1; }

void pfb_sim3d_destroy(pfb_sim3d* s) { delete s; }

int pfb_sim3d_measure_wall(pfb_sim3d* s) {
    if (!s) return set_error(PFB_E_ARG, "null sim");
    if (!hard_wall_channel(s->p.boundary_flags) || !s->d_wall_psi)
        return set_error(PFB_E_CONFIG, "wall diagnostics need the hard-wall channel");
    PFB3_CU(cudaSetDevice(s->device), "cudaSetDevice");
    const float* wide = nullptr;
    PFB3_RC(wide_pool(s, &wide));
    k_wall_diag3d<<<s->N, kWallThreads, 0, s->stream>>>(wide, s->d_cube[s->cur_cube],
                                                       s->d_cells, s->B,
                                                       s->p.Nz, s->p.channel_padding,
                                                       s->p.channel_height, s->d_wall_psi);
    PFB3_CU(cudaGetLastError(), "wall diagnostics");
    PFB3_CU(cudaStreamSynchronize(s->stream), "wall diagnostics");
    return PFB_OK;
}

int pfb_sim3d_verify(pfb_sim3d* s, double* max_rel_V, uint32_t* max_S,
                     unsigned long long* edge_voxels) {
    if (!s || !max_rel_V || !max_S || !edge_voxels) return set_error(PFB_E_ARG, "verify: null argument");
    PFB3_RC(pfb_sim3d_measure_current(s));
    const size_t N = (size_t)s->N;
    Verify3* d_r = nullptr;
    uint32_t* d_m = nullptr;
    std::vector<Verify3> r(N);
    std::vector<pfb_cell3d> c(N);
    int rc = PFB_OK;
    const bool periodic = !substrate_slab(s->p.boundary_flags) && !hard_wall_channel(s->p.boundary_flags);
    if (cudaMalloc(&d_r, N * sizeof(Verify3)) != cudaSuccess || cudaMalloc(&d_m, sizeof(uint32_t)) != cudaSuccess ||
        cudaMemsetAsync(d_m, 0, 4, s->stream) != cudaSuccess) {
        rc = set_error(PFB_E_CUDA, "verify: allocation failed");
    } else {
        const float* wide = nullptr;
        if (wide_pool(s, &wide)) return PFB_E_CUDA;
        k_verify3d<<<s->N, kWallThreads, 0, s->stream>>>(wide, s->d_cube[s->cur_cube],
                                                         s->d_cells, s->B, s->p.Nz,
                                                         periodic ? 1 : 0,
                                                         substrate_slab(s->p.boundary_flags) ? 1 : 0, d_r);
        k_max_u32<<<148, 256, 0, s->stream>>>(s->d_S[s->cur_S], s->s_words, d_m);
        if (cudaGetLastError() != cudaSuccess ||
            cudaMemcpyAsync(r.data(), d_r, N * sizeof(Verify3), cudaMemcpyDeviceToHost, s->stream) != cudaSuccess ||
            cudaMemcpyAsync(c.data(), s->d_cells, N * sizeof(pfb_cell3d), cudaMemcpyDeviceToHost, s->stream) !=
                cudaSuccess ||
            cudaMemcpyAsync(max_S, d_m, 4, cudaMemcpyDeviceToHost, s->stream) != cudaSuccess ||
            cudaStreamSynchronize(s->stream) != cudaSuccess)
            rc = set_error(PFB_E_CUDA, "verify: kernels or readback failed");
    }
    cudaFree(d_r);
    cudaFree(d_m);
    if (rc) return rc;
    double mr = 0.0;
    unsigned long long edges = 0;
    for (size_t i = 0; i < N; ++i) {
        if (r[i].nonfinite) return set_error(PFB_E_STATE, "verify: non-finite sample in cell slot %zu", i);
        mr = std::max(mr, std::fabs(r[i].V - c[i].V) / std::max(1.0, std::fabs(r[i].V)));
        edges += r[i].edge;
    }
    *max_rel_V = mr;
    *edge_voxels = edges;
    return PFB_OK;
}

int pfb_sim3d_boundary_open(pfb_sim3d* s, const char* path, int projection, long long interval,
                            int compress) {
    if (!s) return set_error(PFB_E_ARG, "null sim");
    if (s->bnd) return set_error(PFB_E_STATE, "a boundary recorder is already open");
    PFB3_CU(cudaSetDevice(s->device), "cudaSetDevice");
    s->bnd = pfb::boundary3d_open(path, s->p, projection, interval, compress);
    return s->bnd ? PFB_OK : PFB_E_ARG;
}

int pfb_sim3d_boundary_capture(pfb_sim3d* s) {
    if (!s || !s->bnd) return set_error(PFB_E_STATE, "no boundary recorder is open");
    PFB3_CU(cudaSetDevice(s->device), "cudaSetDevice");
    const float* wide = nullptr;
    PFB3_RC(wide_pool(s, &wide));
    return pfb::boundary3d_capture(s->bnd, wide, s->d_cube[s->cur_cube], s->d_cells, s->B,
                                   s->stream,
                              s->steps_done, (double)s->steps_done * s->p.dt);
}

int pfb_sim3d_boundary_close(pfb_sim3d* s, int complete) {
    if (!s || !s->bnd) return set_error(PFB_E_STATE, "no boundary recorder is open");
    const int rc = pfb::boundary3d_close(s->bnd, complete);
    s->bnd = nullptr;
    return rc;
}

int pfb_sim3d_measure_current(pfb_sim3d* s) {
    if (!s) return set_error(PFB_E_ARG, "null sim");
    PFB3_CU(cudaSetDevice(s->device), "cudaSetDevice");
    PFB3_RC(refresh(s, true, true));
    PFB3_CU(cudaStreamSynchronize(s->stream), "measure_current");
    return PFB_OK;
}

int pfb_sim3d_advance(pfb_sim3d* s, int steps) {
    if (!s || steps < 0) return set_error(PFB_E_ARG, "invalid advance arguments");
    PFB3_CU(cudaSetDevice(s->device), "cudaSetDevice");
    return advance_impl(s, steps);
}

int pfb_sim3d_set_fused(pfb_sim3d* s, int fused) {
    if (!s) return set_error(PFB_E_ARG, "null sim");
    if (fused && step3d_cluster(s->B) == 0)
        return set_error(PFB_E_CONFIG, "brick edge %d does not fit the fused step", s->B);
    if (fused && (s->store || s->mem_mode))
        return set_error(PFB_E_CONFIG, "the fused step needs binary32 pools in the throughput mode");
    const int f = fused ? 1 : 0;
    if (f != s->fused) {
        PFB3_CU(cudaStreamSynchronize(s->stream), "sync");
        s->drop_graph();
        s->fused = f;
    }
    return PFB_OK;
}

int pfb_sim3d_fused(const pfb_sim3d* s) { return s ? s->fused : -1; }

int pfb_sim3d_set_order(pfb_sim3d* s, int morton) {
    if (!s) return set_error(PFB_E_ARG, "null sim");
    PFB3_CU(cudaSetDevice(s->device), "cudaSetDevice");
    s->use_order = morton != 0;
    return refresh_order(s);
}

int pfb_sim3d_set_graph(pfb_sim3d* s, int use_graph) {
    if (!s) return set_error(PFB_E_ARG, "null sim");
    PFB3_CU(cudaStreamSynchronize(s->stream), "sync");
    s->drop_graph();
    s->use_graph = use_graph != 0;
    return PFB_OK;
}

int pfb_sim3d_sync(pfb_sim3d* s) {
    if (!s) return set_error(PFB_E_ARG, "null sim");
    PFB3_CU(cudaStreamSynchronize(s->stream), "sync");
    return PFB_OK;
}

int pfb_sim3d_brick(const pfb_sim3d* s) { return s ? s->B : -1; }

long long pfb_sim3d_step(const pfb_sim3d* s) {
    if (!s) return -1;
    uint64_t v = 0;
    // the driver's stream does not order with the legacy stream: finish it first
    if (cudaStreamSynchronize(s->stream) != cudaSuccess) return -1;
    if (cudaMemcpy(&v, s->d_step, sizeof(v), cudaMemcpyDeviceToHost) != cudaSuccess) return -1;
    return (long long)v;
}

int pfb_sim3d_get_cells(pfb_sim3d* s, pfb_cell3d* out) {
    if (!s || !out) return set_error(PFB_E_ARG, "null argument");
    PFB3_CU(cudaStreamSynchronize(s->stream), "sync");
    PFB3_CU(cudaMemcpy(out, s->d_cells, (size_t)s->N * sizeof(pfb_cell3d), cudaMemcpyDeviceToHost),
            "copy cells");
    return PFB_OK;
}

int pfb_sim3d_get_phi(pfb_sim3d* s, float* out) {
    if (!s || !out) return set_error(PFB_E_ARG, "null argument");
    const float* wide = nullptr;
    PFB3_RC(wide_pool(s, &wide));
    PFB3_CU(cudaStreamSynchronize(s->stream), "sync");
    PFB3_CU(cudaMemcpy(out, wide, (size_t)s->N * s->cell_words * sizeof(float), cudaMemcpyDeviceToHost),
            "copy phi");
    return PFB_OK;
}

int pfb_sim3d_packed_words(pfb_sim3d* s, unsigned long long* words) {
    if (!s || !words) return set_error(PFB_E_ARG, "null argument");
    std::vector<pfb_cell3d> c((size_t)s->N);
    PFB3_RC(pfb_sim3d_get_cells(s, c.data()));
    *words = packed_words(s, c);
    return PFB_OK;
}

int pfb_sim3d_get_packed(pfb_sim3d* s, float* out) {
    if (!s || !out) return set_error(PFB_E_ARG, "null argument");
    std::vector<pfb_cell3d> c((size_t)s->N);
    PFB3_RC(pfb_sim3d_get_cells(s, c.data()));
    const float* wide = nullptr;
    PFB3_RC(wide_pool(s, &wide));
    PFB3_CU(cudaStreamSynchronize(s->stream), "sync");
    size_t off = 0;
    for (int n = 0; n < s->N; ++n) {
        const int E = edge_of(s, c[(size_t)n]);
        const size_t words = (size_t)E * E * E;
        const float* src = E > s->B ? s->h_cube[s->cur_cube][(size_t)n] : wide + (size_t)n * s->cell_words;
        if (!src) return set_error(PFB_E_STATE, "cell %d has no cube of edge %d", n, E);
        PFB3_CU(cudaMemcpy(out + off, src, words * sizeof(float), cudaMemcpyDeviceToHost), "copy field");
        off += words;
    }
    return PFB_OK;
}

int pfb_sim3d_promoted_count(const pfb_sim3d* s) { return s ? s->prom_count() : -1; }

int pfb_sim3d_max_edge(const pfb_sim3d* s) { return s ? s->max_edge : -1; }

long long pfb_sim3d_recoveries(const pfb_sim3d* s) { return s ? s->recoveries : -1; }

int pfb_sim3d_get_S(pfb_sim3d* s, uint32_t* out) {
    if (!s || !out) return set_error(PFB_E_ARG, "null argument");
    PFB3_CU(cudaStreamSynchronize(s->stream), "sync");
    PFB3_CU(cudaMemcpy(out, s->d_S[s->cur_S], s->s_words * sizeof(uint32_t), cudaMemcpyDeviceToHost),
            "copy S");
    return PFB_OK;
}

int pfb_sim3d_get_flags(pfb_sim3d* s, uint32_t* out10) {
    if (!s || !out10) return set_error(PFB_E_ARG, "null argument");
    PFB3_CU(cudaStreamSynchronize(s->stream), "sync");
    PFB3_CU(cudaMemcpy(out10, s->d_flags, PFB3D_FLAG_COUNT * sizeof(uint32_t), cudaMemcpyDeviceToHost),
            "copy flags");
    return PFB_OK;
}

int pfb_sim3d_layout(const pfb_sim3d* s, pfb_layout3d* out) {
    if (!s || !out) return set_error(PFB_E_ARG, "null argument");
    *out = s->L;
    return PFB_OK;
}

int pfb_sim3d_update_args(pfb_sim3d* s, pfb_update_args3d* out) {
    if (!s || !out) return set_error(PFB_E_ARG, "null argument");
    *out = update_args(s);
    return PFB_OK;
}

int pfb_sim3d_measure_args(pfb_sim3d* s, pfb_measure_args3d* out) {
    if (!s || !out) return set_error(PFB_E_ARG, "null argument");
    const bool full = s->p.full_moment_every > 0 && s->steps_done % s->p.full_moment_every == 0;
    *out = measure_args(s, true, full);
    return PFB_OK;
}

void* pfb_sim3d_stream(const pfb_sim3d* s) { return s ? (void*)s->stream : nullptr; }

int pfb_sim3d_bench(pfb_sim3d* s, int warmup, int steps, double* ms) {
    if (!s || warmup < 0 || steps <= 0 || !ms) return set_error(PFB_E_ARG, "invalid bench arguments");
    PFB3_CU(cudaSetDevice(s->device), "cudaSetDevice");
    PFB3_RC(advance_impl(s, warmup));
    cudaEvent_t e0, e1;
    PFB3_CU(cudaEventCreate(&e0), "event");
    PFB3_CU(cudaEventCreate(&e1), "event");
    PFB3_CU(cudaStreamSynchronize(s->stream), "sync");
    PFB3_CU(cudaEventRecord(e0, s->stream), "record");
    PFB3_RC(advance_impl(s, steps));
    PFB3_CU(cudaEventRecord(e1, s->stream), "record");
    PFB3_CU(cudaEventSynchronize(e1), "sync");
    float t = 0.0f;
    PFB3_CU(cudaEventElapsedTime(&t, e0, e1), "elapsed");
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    *ms = (double)t;
    return PFB_OK;
}

}  // extern "C"
