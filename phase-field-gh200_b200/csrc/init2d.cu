// Set-up and diagnostic passes of the 2D path over whole cell tiles: seeding
// of the tanh disks, the initial moments, the Q5.27 aggregate rebuilt from a
// phi pool, the invariant check, the S maximum, the trajectory record pack and
// the 16-bit pool conversions.
//
// Behaviour follows the reference's set-up kernels (src/kernels.cu:1044-1265):
// the seed profile phi = (1 - tanh(k (r - R_eff)))/2 and its origin rounding,
// the Q5.27 overflow and clamp tests, the support threshold and the trajectory
// record's fields. The layout of the work is this file's own:
//
//  * every pass walks a tile as 288 rows of 72 four-pixel chunks (one 16-byte
//    access each); a cell's tile is split into kBands bands of 72 rows, one
//    CTA per band, so a launch has 4 N CTAs and stores are vectorised;
//  * passes that reduce over a cell (moments, invariant check) run the four
//    band CTAs of a cell as one thread-block cluster: each CTA folds its band
//    (warp butterfly, then its warps in order) and pushes the partial into
//    rank 0's shared memory with st.async; rank 0 adds the ranks in order and
//    commits, so the sums are deterministic;
//  * seeding writes both pools in the same pass (disk or zero in pool a,
//    zero in pool b), so no separate clearing sweep runs.
#include <cuda_runtime.h>

#include <cstdint>

#include "device_util.cuh"
#include "pfb_common.cuh"
#include "pfb_internal.h"
#include "storage2d.cuh"

#include <algorithm>

namespace pfb {

namespace {

constexpr int kChunks = kTilePitch / 4;           // 72 four-pixel chunks per tile row
constexpr int kBands = 4;                         // CTAs per cell
constexpr int kBandRows = kTilePitch / kBands;    // 72 tile rows per CTA
constexpr int kPassThreads = 288;                 // 4 tile rows x 72 chunks per sweep
constexpr int kPassWarps = kPassThreads / 32;
constexpr int kRowsPerSweep = kPassThreads / kChunks;
static_assert(kTilePitch % (4 * kBands) == 0 && kPassThreads % kChunks == 0, "tile walk");
static_assert(kBandRows % kRowsPerSweep == 0, "band walk");

__device__ __forceinline__ int fold(int v, int L) {
    v %= L;
    return v < 0 ? v + L : v;
}

// Origin of the class window whose centre pixel lies nearest (cx, cy).
__device__ __forceinline__ int window_origin(float c, int w, int L) {
    return fold((int)lrintf(c - 0.5f * (float)(w - 1)), L);
}

// Seed value of a pixel at lattice position (gx, gy) for the disk at (cx, cy)
// on the periodic lattice of side L.
__device__ __forceinline__ float seed_value(int gx, int gy, float cx, float cy, float L,
                                            float radius_eff, float kappa_iface) {
    const float half = 0.5f * L;
    float dx = (float)gx - cx;
    float dy = (float)gy - cy;
    if (dx > half) dx -= L;
    if (dx < -half) dx += L;
    if (dy > half) dy -= L;
    if (dy < -half) dy += L;
    // the reference's build contracts dx*dx + dy*dy into fma(dx, dx, dy*dy);
    // written out so the seed stays bit-identical whatever the code around it
    const float r = sqrtf(__fmaf_rn(dx, dx, __fmul_rn(dy, dy)));
    return 0.5f * (1.0f - tanhf(kappa_iface * (r - radius_eff)));
}

// ---- seeding -----------------------------------------------------------------
// CTA (band, n): tile rows [band*72, band*72 + 72) of cell n in both pools.
__global__ void __launch_bounds__(kPassThreads)
    k_seed_tiles2d(float* __restrict__ phi_a, float* __restrict__ phi_b,
                   pfb_cell2d* __restrict__ cell, const uint8_t* __restrict__ clsv, int L,
                   const float* __restrict__ seed_cx, const float* __restrict__ seed_cy,
                   float radius_eff, float kappa_iface) {
    const int n = blockIdx.x / kBands, band = blockIdx.x % kBands;
    const int cls = (int)clsv[n];
    const Window w = window_of(cls);
    const float cx = seed_cx[n], cy = seed_cy[n];
    const int gx0 = window_origin(cx, w.wx, L), gy0 = window_origin(cy, w.wy, L);
    float4* ta = reinterpret_cast<float4*>(phi_a + (size_t)n * kTileArea);
    float4* tb = reinterpret_cast<float4*>(phi_b + (size_t)n * kTileArea);
    const int c = threadIdx.x % kChunks;
    const float zero4[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    for (int y = band * kBandRows + threadIdx.x / kChunks; y < (band + 1) * kBandRows;
         y += kRowsPerSweep) {
        const int b = y - w.ty0;
        float v[4] = {zero4[0], zero4[1], zero4[2], zero4[3]};
        if ((unsigned)b < (unsigned)w.wy) {
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int a = 4 * c + j - w.tx0;
                if ((unsigned)a < (unsigned)w.wx)
                    v[j] = seed_value(gx0 + a, gy0 + b, cx, cy, (float)L, radius_eff,
                                      kappa_iface);
            }
        }
        const size_t i = (size_t)y * kChunks + c;
        ta[i] = make_float4(v[0], v[1], v[2], v[3]);
        tb[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    }
    if (band == 0 && threadIdx.x == 0) {
        pfb_cell2d& cs = cell[n];
        cs.gx0 = gx0;
        cs.gy0 = gy0;
        cs.cls = (uint8_t)cls;
        cs.cls_written[0] = (uint8_t)cls;
        cs.cls_written[1] = (uint8_t)cls;
    }
}

// ---- cluster fold of per-thread partials ---------------------------------------
// ND doubles (summed) and NI ints (NI_MIN folded by min, the rest by max) of
// every thread of the cluster arrive in rank 0, in a fixed order.
template <int ND, int NI, int NI_MIN>
struct Fold {
    uint64_t bar;
    double wd[kPassWarps][ND];
    int wi[kPassWarps][NI];
    alignas(16) double rd[kBands][ND];
    alignas(16) int ri[kBands][NI];
    static_assert(ND % 2 == 0 && NI % 4 == 0, "vector pushes");

    // thread 0 of every CTA, before the cluster's first barrier
    __device__ void init(int rank) {
        dev::mbar_init(&bar, 1);
        if (rank == 0)
            dev::mbar_arrive_expect_tx(&bar, (uint32_t)(kBands * (8 * ND + 4 * NI)));
    }

    // All threads of all CTAs call it; returns true in lane 0 of warp 0 of
    // rank 0, with the cluster totals in d and i.
    __device__ bool run(int rank, double (&d)[ND], int (&i)[NI], uint32_t* status) {
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
        for (int k = 0; k < ND; ++k) d[k] = dev::warp_sum_down(d[k]);
#pragma unroll
        for (int k = 0; k < NI; ++k)
            i[k] = k < NI_MIN ? dev::warp_min_down(i[k]) : dev::warp_max_down(i[k]);
        if (lane == 0) {
#pragma unroll
            for (int k = 0; k < ND; ++k) wd[warp][k] = d[k];
#pragma unroll
            for (int k = 0; k < NI; ++k) wi[warp][k] = i[k];
        }
        __syncthreads();
        dev::cluster_wait();  // rank 0's barrier is initialised
        if (warp != 0) return false;
        double s[ND];
#pragma unroll
        for (int k = 0; k < ND; ++k)
            s[k] = dev::ordered_lane_sum(lane < kPassWarps ? wd[lane][k] : 0.0, kPassWarps);
        int m[NI];
#pragma unroll
        for (int k = 0; k < NI; ++k) {
            const int x = lane < kPassWarps ? wi[lane][k] : wi[0][k];
            m[k] = k < NI_MIN ? __reduce_min_sync(0xFFFFFFFFu, x) : __reduce_max_sync(0xFFFFFFFFu, x);
        }
        if (lane == 0) {
            const uint32_t b = dev::map_to_rank(dev::smem_addr(&bar), 0);
#pragma unroll
            for (int k = 0; k < ND; k += 2)
                dev::st_async_v2f64(dev::map_to_rank(dev::smem_addr(&rd[rank][k]), 0), s[k],
                                    s[k + 1], b);
#pragma unroll
            for (int k = 0; k < NI; k += 4)
                dev::st_async_v4b32(dev::map_to_rank(dev::smem_addr(&ri[rank][k]), 0), m[k],
                                    m[k + 1], m[k + 2], m[k + 3], b);
        }
        if (rank != 0) return false;
        if (!dev::mbar_wait_bounded(&bar, 0, 1u << 24)) {
            if (lane == 0) atomicOr(status, 1u);
            return false;
        }
#pragma unroll
        for (int k = 0; k < ND; ++k)
            d[k] = dev::ordered_lane_sum(lane < kBands ? rd[lane][k] : 0.0, kBands);
#pragma unroll
        for (int k = 0; k < NI; ++k) {
            const int x = lane < kBands ? ri[lane][k] : ri[0][k];
            i[k] = k < NI_MIN ? __reduce_min_sync(0xFFFFFFFFu, x) : __reduce_max_sync(0xFFFFFFFFu, x);
        }
        return lane == 0;
    }
};

// Status word of these passes: bit 0 = a cluster fold gave up waiting.
__device__ unsigned int g_init2d_status = 0u;

// ---- initial moments -----------------------------------------------------------
// V, Cx, Cy (window coordinates), support box and phi_max of the window;
// clears the demotion counter and the interaction integral.
__global__ void __launch_bounds__(kPassThreads)
    k_window_moments2d(pfb_cell2d* __restrict__ cell, const uint8_t* __restrict__ clsv,
                       const float* __restrict__ phi) {
    __shared__ Fold<4, 8, 2> F;  // d: V Cx Cy pad; i: lo_x lo_y | hi_x hi_y pmax pad...
    const int n = blockIdx.x / kBands;
    const int rank = (int)dev::cluster_rank();
    if (threadIdx.x == 0) F.init(rank);
    dev::cluster_arrive_relaxed();
    const Window w = window_of((int)clsv[n]);
    const float4* t = reinterpret_cast<const float4*>(phi + (size_t)n * kTileArea);
    const int c = threadIdx.x % kChunks;
    double d[4] = {0.0, 0.0, 0.0, 0.0};
    int i[8] = {w.wx, w.wy, -1, -1, 0, 0, 0, 0};
    for (int y = rank * kBandRows + threadIdx.x / kChunks; y < (rank + 1) * kBandRows;
         y += kRowsPerSweep) {
        const int b = y - w.ty0;
        if ((unsigned)b >= (unsigned)w.wy) continue;
        const float4 q = __ldg(t + (size_t)y * kChunks + c);
        const float v[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int a = 4 * c + j - w.tx0;
            if ((unsigned)a >= (unsigned)w.wx) continue;
            const double s = (double)v[j] * (double)v[j];
            d[0] += s;
            d[1] += s * (double)a;
            d[2] += s * (double)b;
            i[4] = max(i[4], (int)__float_as_uint(fabsf(v[j])));
            if (v[j] > kSupportEps) {
                i[0] = min(i[0], a);
                i[1] = min(i[1], b);
                i[2] = max(i[2], a);
                i[3] = max(i[3], b);
            }
        }
    }
    if (F.run(rank, d, i, &g_init2d_status)) {
        pfb_cell2d& cs = cell[n];
        cs.V = d[0];
        cs.Cx = d[1];
        cs.Cy = d[2];
        cs.bb_lo_x = i[0];
        cs.bb_lo_y = i[1];
        cs.bb_hi_x = i[2];
        cs.bb_hi_y = i[3];
        cs.phi_max = __uint_as_float((uint32_t)i[4]);
        cs.promote_ctr = 0u;
        cs.Ix = 0.0;
        cs.Iy = 0.0;
    }
}

// ---- invariant check ---------------------------------------------------------------
// out_V[n] = sum of phi^2 over the window; out_outside[n] = max |phi| over the
// tile outside the window (the tile invariant wants 0; NaN samples are passed
// over there, as the reference's fmaxf fold does).
__global__ void __launch_bounds__(kPassThreads)
    k_window_verify2d(const float* __restrict__ phi, const uint8_t* __restrict__ clsv,
                      double* __restrict__ out_V, float* __restrict__ out_outside) {
    __shared__ Fold<2, 4, 0> F;  // d: V pad; i: max |phi| bits outside, pad
    const int n = blockIdx.x / kBands;
    const int rank = (int)dev::cluster_rank();
    if (threadIdx.x == 0) F.init(rank);
    dev::cluster_arrive_relaxed();
    const Window w = window_of((int)clsv[n]);
    const float4* t = reinterpret_cast<const float4*>(phi + (size_t)n * kTileArea);
    const int c = threadIdx.x % kChunks;
    double d[2] = {0.0, 0.0};
    int i[4] = {0, 0, 0, 0};
    for (int y = rank * kBandRows + threadIdx.x / kChunks; y < (rank + 1) * kBandRows;
         y += kRowsPerSweep) {
        const bool row_in = (unsigned)(y - w.ty0) < (unsigned)w.wy;
        const float4 q = __ldg(t + (size_t)y * kChunks + c);
        const float v[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            if (row_in && (unsigned)(4 * c + j - w.tx0) < (unsigned)w.wx)
                d[0] += (double)v[j] * (double)v[j];
            else if (!isnan(v[j]))  // |phi| bit patterns order like the values
                i[0] = max(i[0], (int)__float_as_uint(fabsf(v[j])));
        }
    }
    if (F.run(rank, d, i, &g_init2d_status)) {
        out_V[n] = d[0];
        out_outside[n] = __uint_as_float((uint32_t)i[0]);
    }
}

// ---- aggregate rebuild ------------------------------------------------------------
// CTA (band, n) adds q(phi) of its window rows into S at the cell's lattice
// position; an add that wraps the 32-bit word raises S_overflow, a clamped
// square raises q_clamp.
__global__ void __launch_bounds__(kPassThreads)
    k_window_scatter2d(const float* __restrict__ phi, const pfb_cell2d* __restrict__ cell,
                       const uint8_t* __restrict__ clsv, uint32_t* __restrict__ S, int L, int P,
                       uint32_t* __restrict__ flags) {
    const int n = blockIdx.x / kBands, band = blockIdx.x % kBands;
    const Window w = window_of((int)clsv[n]);
    const int gx0 = cell[n].gx0, gy0 = cell[n].gy0;
    const float4* t = reinterpret_cast<const float4*>(phi + (size_t)n * kTileArea);
    const int c = threadIdx.x % kChunks;
    bool ovf = false, clamp = false;
    for (int y = band * kBandRows + threadIdx.x / kChunks; y < (band + 1) * kBandRows;
         y += kRowsPerSweep) {
        const int b = y - w.ty0;
        if ((unsigned)b >= (unsigned)w.wy) continue;
        const float4 q4 = __ldg(t + (size_t)y * kChunks + c);
        const float v[4] = {q4.x, q4.y, q4.z, q4.w};
        uint32_t* srow = S + (size_t)fold(gy0 + b, L) * P;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int a = 4 * c + j - w.tx0;
            if ((unsigned)a >= (unsigned)w.wx) continue;
            const uint32_t q = q_encode(v[j]);
            if (!q) continue;
            int gx = gx0 + a;
            if (gx >= L) gx -= L;
            const uint32_t old = atomicAdd(srow + gx, q);
            ovf |= old > 0xFFFFFFFFu - q;
            clamp |= v[j] * v[j] > kPhiSqCap;
        }
    }
    if (__any_sync(0xFFFFFFFFu, ovf) && (threadIdx.x & 31) == 0)
        atomicOr(flags + PFB_FLAG_S_OVERFLOW, 1u);
    if (__any_sync(0xFFFFFFFFu, clamp) && (threadIdx.x & 31) == 0)
        atomicOr(flags + PFB_FLAG_Q_CLAMP, 1u);
}

// ---- largest aggregate word ----------------------------------------------------------
__global__ void k_max_words(const uint32_t* __restrict__ S, size_t n, uint32_t* out_max) {
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    const size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const size_t n4 = ((uintptr_t)S & 15u) ? 0 : n / 4;
    uint32_t m = 0u;
    const uint4* S4 = reinterpret_cast<const uint4*>(S);
    for (size_t k = tid; k < n4; k += stride) {
        const uint4 v = __ldcs(S4 + k);
        m = max(max(m, max(v.x, v.y)), max(v.z, v.w));
    }
    for (size_t k = 4 * n4 + tid; k < n; k += stride) m = max(m, S[k]);
    m = __reduce_max_sync(0xFFFFFFFFu, m);
    if ((threadIdx.x & 31) == 0 && m) atomicMax(out_max, m);
}

// ---- trajectory records -------------------------------------------------------------
// Periodic centroid in lattice coordinates, x = gx0 + Cx / V wrapped into
// [0, L) (V <= 0 is read as 1), with the record's other fields.
__device__ __forceinline__ pfb_traj_cell2d traj_record(const pfb_cell2d& cs, int cls, int L) {
    const double vol = cs.V > 0.0 ? cs.V : 1.0;
    const double px = (double)cs.gx0 + cs.Cx / vol;
    const double py = (double)cs.gy0 + cs.Cy / vol;
    pfb_traj_cell2d r;
    r.global_id = cs.global_id;
    r.cls = (int32_t)cls;
    r.cx = (float)(px - floor(px / (double)L) * (double)L);
    r.cy = (float)(py - floor(py / (double)L) * (double)L);
    r.vx = cs.vx;
    r.vy = cs.vy;
    r.theta = cs.theta;
    r.volume = (float)cs.V;
    r.perim = (float)cs.perim;
    r.gamma = cs.gamma;
    r.v_A = cs.v_A;
    r.phi_max = cs.phi_max;
    return r;
}

__global__ void k_pack_traj2d(const pfb_cell2d* __restrict__ cell, const uint8_t* __restrict__ clsv,
                              pfb_traj_cell2d* __restrict__ out, int N, int L) {
    for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < N; n += gridDim.x * blockDim.x)
        out[n] = traj_record(cell[n], (int)clsv[n], L);
}

// Trajectory frames written by the device straight into page-locked host
// memory (the records of one frame leave each CTA as consecutive 16-byte
// chunks, so the host link sees full-width writes). Every CTA reads the
// ring's frame counter first; the last CTA to finish advances it, so frames
// follow each other in stream order, graph replays included.
constexpr int kRingThreads = 128;
static_assert(sizeof(pfb_traj_cell2d) == 48, "trajectory record is three 16-byte chunks");

__global__ void k_ring_begin(TrajRing2D* r, pfb_traj_cell2d* base, int frames) {
    r->base = base;
    r->frames = frames;
    r->k = 0ull;
    r->arrived = 0u;
}

__global__ void __launch_bounds__(kRingThreads)
    k_pack_traj2d_ring(const pfb_cell2d* __restrict__ cell, const uint8_t* __restrict__ clsv,
                       TrajRing2D* ring, int N, int L) {
    __shared__ uint4 stage[kRingThreads * 3];
    const TrajRing2D rg = *ring;
    uint4* dst = reinterpret_cast<uint4*>(rg.base + (size_t)(rg.k % (unsigned long long)rg.frames) * N);
    for (int n0 = (int)blockIdx.x * kRingThreads; n0 < N; n0 += (int)gridDim.x * kRingThreads) {
        const int n = n0 + (int)threadIdx.x;
        if (n < N) reinterpret_cast<pfb_traj_cell2d*>(stage)[threadIdx.x] = traj_record(cell[n], (int)clsv[n], L);
        __syncthreads();
        const int chunks = 3 * min(kRingThreads, N - n0);
        for (int i = (int)threadIdx.x; i < chunks; i += kRingThreads) dst[(size_t)3 * n0 + i] = stage[i];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(&ring->arrived, 1u) == gridDim.x - 1) {
            ring->arrived = 0u;
            ring->k = rg.k + 1ull;
        }
    }
}

// The same for many systems in one launch: global record g belongs to the
// last system r with src[r].off <= g; the frame holds `total` records.
__global__ void __launch_bounds__(kRingThreads)
    k_pack_traj2d_ring_batch(const TrajSource2D* __restrict__ src, int R, int total, TrajRing2D* ring) {
    __shared__ uint4 stage[kRingThreads * 3];
    const TrajRing2D rg = *ring;
    uint4* dst = reinterpret_cast<uint4*>(rg.base + (size_t)(rg.k % (unsigned long long)rg.frames) * total);
    for (int g0 = (int)blockIdx.x * kRingThreads; g0 < total; g0 += (int)gridDim.x * kRingThreads) {
        const int g = g0 + (int)threadIdx.x;
        if (g < total) {
            int lo = 0, hi = R - 1;
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (src[mid].off <= g)
                    lo = mid;
                else
                    hi = mid - 1;
            }
            const TrajSource2D& t = src[lo];
            const int n = g - t.off;
            reinterpret_cast<pfb_traj_cell2d*>(stage)[threadIdx.x] = traj_record(t.cell[n], (int)t.cls[n], t.L);
        }
        __syncthreads();
        const int chunks = 3 * min(kRingThreads, total - g0);
        for (int i = (int)threadIdx.x; i < chunks; i += kRingThreads) dst[(size_t)3 * g0 + i] = stage[i];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(&ring->arrived, 1u) == gridDim.x - 1) {
            ring->arrived = 0u;
            ring->k = rg.k + 1ull;
        }
    }
}

int launch_status(const char* what) {
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return set_error(PFB_E_CUDA, "%s: %s", what, cudaGetErrorString(e));
    return PFB_OK;
}

// Launch of a per-cell cluster pass: N clusters of kBands CTAs.
template <typename... Args>
cudaError_t launch_cluster_pass(void (*kern)(Args...), int N, cudaStream_t s, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(N * kBands), 1, 1);
    cfg.blockDim = dim3(kPassThreads, 1, 1);
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = kBands;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kern, args...);
}

}  // namespace

int init_tiles2d(float* phi_a, float* phi_b, pfb_cell2d* cell, const uint8_t* cls, int N, int L,
                 const float* cx, const float* cy, float radius_eff, float kappa_iface,
                 cudaStream_t s) {
    if (!phi_a || !phi_b || !cell || !cls || !cx || !cy || N < 0 || L <= 0)
        return set_error(PFB_E_ARG, "init_tiles2d: bad argument");
    if (((uintptr_t)phi_a | (uintptr_t)phi_b) & 15u)
        return set_error(PFB_E_ARG, "init_tiles2d: pools must be 16-byte aligned");
    if (N == 0) return PFB_OK;
    k_seed_tiles2d<<<N * kBands, kPassThreads, 0, s>>>(phi_a, phi_b, cell, cls, L, cx, cy,
                                                       radius_eff, kappa_iface);
    return launch_status("init_tiles2d");
}

int init_moments2d(pfb_cell2d* cell, const uint8_t* cls, const float* phi, int N, cudaStream_t s) {
    if (!cell || !cls || !phi || N < 0) return set_error(PFB_E_ARG, "init_moments2d: bad argument");
    if ((uintptr_t)phi & 15u) return set_error(PFB_E_ARG, "init_moments2d: pool must be 16-byte aligned");
    if (N == 0) return PFB_OK;
    const cudaError_t e = launch_cluster_pass(k_window_moments2d, N, s, cell, cls, phi);
    if (e != cudaSuccess) return set_error(PFB_E_CUDA, "init_moments2d: %s", cudaGetErrorString(e));
    return PFB_OK;
}

int scatter_all2d(const float* phi, const pfb_cell2d* cell, const uint8_t* cls, uint32_t* S,
                  int N, int L, int P, uint32_t* flags, cudaStream_t s) {
    if (!phi || !cell || !cls || !S || !flags || N < 0 || L <= 0 || P < L)
        return set_error(PFB_E_ARG, "scatter_all2d: bad argument");
    if ((uintptr_t)phi & 15u) return set_error(PFB_E_ARG, "scatter_all2d: pool must be 16-byte aligned");
    if (N == 0) return PFB_OK;
    k_window_scatter2d<<<N * kBands, kPassThreads, 0, s>>>(phi, cell, cls, S, L, P, flags);
    return launch_status("scatter_all2d");
}

int zero_u32(uint32_t* p, size_t n, cudaStream_t s) {
    if (!p && n) return set_error(PFB_E_ARG, "zero_u32: null");
    if (!n) return PFB_OK;
    const cudaError_t e = cudaMemsetAsync(p, 0, n * sizeof(uint32_t), s);
    if (e != cudaSuccess) return set_error(PFB_E_CUDA, "zero_u32: %s", cudaGetErrorString(e));
    return PFB_OK;
}

int verify_cells2d(const float* phi, const pfb_cell2d* cell, const uint8_t* cls, int N,
                   double* out_V, float* out_outside, cudaStream_t s) {
    if (!phi || !cell || !cls || !out_V || !out_outside || N < 0)
        return set_error(PFB_E_ARG, "verify_cells2d: bad argument");
    if ((uintptr_t)phi & 15u) return set_error(PFB_E_ARG, "verify_cells2d: pool must be 16-byte aligned");
    if (N == 0) return PFB_OK;
    const cudaError_t e = launch_cluster_pass(k_window_verify2d, N, s, phi, cls, out_V, out_outside);
    if (e != cudaSuccess) return set_error(PFB_E_CUDA, "verify_cells2d: %s", cudaGetErrorString(e));
    return PFB_OK;
}

int verify_S(const uint32_t* S, size_t n, uint32_t* out_max, cudaStream_t s) {
    if (!S || !out_max) return set_error(PFB_E_ARG, "verify_S: null");
    if (!n) return PFB_OK;
    const size_t want = (n / 4 + 255) / 256;
    k_max_words<<<(unsigned)std::max<size_t>(1, std::min<size_t>(want, 148 * 8)), 256, 0, s>>>(
        S, n, out_max);
    return launch_status("verify_S");
}

int pack_traj2d(const pfb_cell2d* cell, const uint8_t* cls, pfb_traj_cell2d* out, int N, int L,
                cudaStream_t s) {
    if (!cell || !cls || !out || N < 0 || L <= 0) return set_error(PFB_E_ARG, "pack_traj2d: bad argument");
    if (N == 0) return PFB_OK;
    k_pack_traj2d<<<std::min((N + 127) / 128, 148 * 4), 128, 0, s>>>(cell, cls, out, N, L);
    return launch_status("pack_traj2d");
}

int ring_begin2d(TrajRing2D* ring, pfb_traj_cell2d* base, int frames, cudaStream_t s) {
    if (!ring || !base || frames < 1 || ((uintptr_t)base & 15u))
        return set_error(PFB_E_ARG, "ring_begin2d: bad argument");
    k_ring_begin<<<1, 1, 0, s>>>(ring, base, frames);
    return launch_status("ring_begin2d");
}

int pack_traj2d_ring(const pfb_cell2d* cell, const uint8_t* cls, TrajRing2D* ring, int N, int L,
                     cudaStream_t s) {
    if (!cell || !cls || !ring || N < 1 || L <= 0) return set_error(PFB_E_ARG, "pack_traj2d_ring: bad argument");
    k_pack_traj2d_ring<<<std::min((N + kRingThreads - 1) / kRingThreads, 148), kRingThreads, 0, s>>>(
        cell, cls, ring, N, L);
    return launch_status("pack_traj2d_ring");
}

int pack_traj2d_ring_batch(const TrajSource2D* src, int R, int total, TrajRing2D* ring, cudaStream_t s) {
    if (!src || R < 1 || total < 1 || !ring) return set_error(PFB_E_ARG, "pack_traj2d_ring_batch: bad argument");
    k_pack_traj2d_ring_batch<<<std::min((total + kRingThreads - 1) / kRingThreads, 148), kRingThreads, 0, s>>>(
        src, R, total, ring);
    return launch_status("pack_traj2d_ring_batch");
}

int init2d_read_status(unsigned* out, int clear) {
    unsigned v = 0;
    cudaError_t e = cudaMemcpyFromSymbol(&v, g_init2d_status, sizeof(v));
    if (e != cudaSuccess) return set_error(PFB_E_CUDA, "status read: %s", cudaGetErrorString(e));
    if (clear) {
        const unsigned z = 0;
        e = cudaMemcpyToSymbol(g_init2d_status, &z, sizeof(z));
        if (e != cudaSuccess) return set_error(PFB_E_CUDA, "status clear: %s", cudaGetErrorString(e));
    }
    if (out) *out = v;
    return PFB_OK;
}

}  // namespace pfb

// ---- 16-bit phi pools: conversions at the host boundary -------------------
namespace pfb {

__global__ void k_narrow_pool(const float* __restrict__ in, uint16_t* __restrict__ out, size_t n,
                              int storage) {
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        out[i] = storage == kStoreF16 ? __half_as_ushort(__float2half_rn(in[i]))
                                      : __bfloat16_as_ushort(__float2bfloat16_rn(in[i]));
}

__global__ void k_widen_pool(const uint16_t* __restrict__ in, float* __restrict__ out, size_t n,
                             int storage) {
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        out[i] = storage == kStoreF16 ? Store<__half>::value(in[i])
                                      : Store<__nv_bfloat16>::value(in[i]);
}

int narrow_pool(const float* in, void* out, size_t n, int storage, cudaStream_t s) {
    if (!in || !out) return set_error(PFB_E_ARG, "narrow_pool: null");
    const int blocks = (int)std::min<size_t>(148 * 8, (n + 255) / 256 + 1);
    k_narrow_pool<<<blocks, 256, 0, s>>>(in, static_cast<uint16_t*>(out), n, storage);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? PFB_OK : set_error(PFB_E_CUDA, "narrow_pool: %s", cudaGetErrorString(e));
}

int widen_pool(const void* in, float* out, size_t n, int storage, cudaStream_t s) {
    if (!in || !out) return set_error(PFB_E_ARG, "widen_pool: null");
    const int blocks = (int)std::min<size_t>(148 * 8, (n + 255) / 256 + 1);
    k_widen_pool<<<blocks, 256, 0, s>>>(static_cast<const uint16_t*>(in), out, n, storage);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? PFB_OK : set_error(PFB_E_CUDA, "widen_pool: %s", cudaGetErrorString(e));
}

}  // namespace pfb
