// Velocity observation of the 2D step: the independent dense observer and
// the PFVMOM4 velocity-component recorder (reference src/velocity_moments.cu,
// src/velocity_output.cu, include/velocity_sampling.hpp,
// common/velocity_moments.h, common/velocity_format.h).
//
// The fused observers live in the step kernel (OBS template of k_step2d):
// advection steps integrate the velocity components into each cell's
// `advection` record; spatial steps also measure the passive interfacial and
// overlap rates and hold them until the next spatial sample. The recorder
// decides per step which observer runs, and at each frame closes the held
// intervals on the host with the rates of an independent dense pass over the
// current field.
#include <cuda_runtime.h>

#include <cerrno>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "device_util.cuh"
#include "pfb200_ckpt.h"
#include "pfb_common.cuh"
#include "pfb_internal.h"

namespace pfb {
namespace {

constexpr int kColumns = 26;        // PFVMOM4 columns per cell
constexpr int kIntegralColumn = 9;  // q[0..11]
constexpr int kSpatialCountColumn = 21;
constexpr int kEndpointColumn = 22;

// ---- the dense observer -------------------------------------------------------
// One thread-block cluster of kObsBands CTAs per cell. CTA r walks tile rows
// [72 r, 72 r + 72) as four-pixel chunks (288 threads: 4 rows x 72 chunks per
// sweep); samples outside the cell's class window read as zero. Two passes:
//   1. the interaction integral of phi^n, pushed by every CTA into every
//      CTA's shared memory (st.async) and summed there in rank order, so all
//      CTAs derive the same velocity;
//   2. the eight centroid-moment channels, pushed into rank 0, which adds them
//      in rank order and commits the rates times dt.
constexpr int kObsBands = 4;
constexpr int kObsThreads = 288;
constexpr int kObsWarps = kObsThreads / 32;
constexpr int kObsChunks = kTilePitch / 4;
constexpr int kObsBandRows = kTilePitch / kObsBands;
constexpr int kObsSweep = kObsThreads / kObsChunks;
static_assert(kObsBandRows % kObsSweep == 0, "band walk");

struct ObsShared {
    uint64_t barF;  // kObsBands force partials (16 B each), every CTA
    uint64_t barM;  // kObsBands channel partials (64 B each), rank 0
    double wf[kObsWarps][2];
    double wm[kObsWarps][8];
    alignas(16) double rf[kObsBands][2];
    alignas(16) double rm[kObsBands][8];
    double vel[4];
};

// Three rows (y-1, y, y+1) of a four-pixel chunk with its left and right
// neighbours, window-masked: v[r][k] is tile column 4c - 1 + k of row y - 1 + r.
struct Chunk3 {
    float v[3][6];
};

__device__ __forceinline__ Chunk3 load_chunk(const float* tile, const Window& w, int y, int c) {
    Chunk3 q;
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        const int yy = y - 1 + r;
        const bool row_in = (unsigned)(yy - w.ty0) < (unsigned)w.wy;
        const float* row = tile + (size_t)yy * kTilePitch;
        const float4 mid = row_in ? __ldg(reinterpret_cast<const float4*>(row) + c)
                                  : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        const float m4[4] = {mid.x, mid.y, mid.z, mid.w};
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            const int x = 4 * c - 1 + k;
            const bool in = row_in && (unsigned)(x - w.tx0) < (unsigned)w.wx;
            q.v[r][k] = !in ? 0.0f : (k >= 1 && k <= 4) ? m4[k - 1] : __ldg(row + x);
        }
    }
    return q;
}

// S_other at window pixel (a, b) of a cell holding p there; an aggregate below
// the cell's own share reads as NaN, so that a frame built from it is refused.
__device__ __forceinline__ float other_share(const pfb_step_args2d& A, const pfb_cell2d& c, int a,
                                             int b, float p) {
    const int gx = (c.gx0 + a) % A.L, gy = (c.gy0 + b) % A.L;
    const uint32_t all = A.S_rd[(size_t)gy * A.P + gx], self = q_encode(p);
    return all >= self ? (float)(all - self) * kQInv : __int_as_float(0x7fc00000);
}

// Warp butterflies, then this CTA's warps in order, into lane 0 of warp 0.
template <int NV>
__device__ __forceinline__ void cta_fold(double (&v)[NV], double (*slots)[NV]) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int j = 0; j < NV; ++j) v[j] = dev::warp_sum_down(v[j]);
    if (lane == 0)
#pragma unroll
        for (int j = 0; j < NV; ++j) slots[warp][j] = v[j];
    __syncthreads();
    if (warp == 0)
#pragma unroll
        for (int j = 0; j < NV; ++j)
            v[j] = dev::ordered_lane_sum(lane < kObsWarps ? slots[lane][j] : 0.0, kObsWarps);
}

// Adds the velocity the step would take (tumble included) and the twelve
// centroid-moment channels of phi^n, each rate times dt, to out[n]
// (the reference's dense observer, src/velocity_moments.cu:43-123).
__global__ void __launch_bounds__(kObsThreads)
    k_observe2d(const __grid_constant__ pfb_step_args2d A, pfb_moment_accum2d* out, double dt) {
    __shared__ ObsShared sh;
    const int n = blockIdx.x / kObsBands;
    const int rank = (int)dev::cluster_rank();
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) {
        dev::mbar_init(&sh.barF, 1);
        dev::mbar_init(&sh.barM, 1);
        dev::mbar_arrive_expect_tx(&sh.barF, kObsBands * 16u);
        if (rank == 0) dev::mbar_arrive_expect_tx(&sh.barM, kObsBands * 64u);
    }
    dev::cluster_arrive_relaxed();
    const pfb_cell2d& c = A.cell[n];
    const Window w = window_of(c.cls);
    const float* tile = A.phi_in + (size_t)n * kTileArea;
    const int ch = tid % kObsChunks;
    const int y_lo = rank * kObsBandRows + tid / kObsChunks, y_hi = (rank + 1) * kObsBandRows;

    // ---- pass 1: interaction integral (binary32 products, FP64 sums)
    double f[2] = {0.0, 0.0};
    for (int y = y_lo; y < y_hi; y += kObsSweep) {
        const int b = y - w.ty0;
        if ((unsigned)b >= (unsigned)w.wy) continue;
        const Chunk3 q = load_chunk(tile, w, y, ch);
#pragma unroll
        for (int k = 1; k <= 4; ++k) {
            const int a = 4 * ch - 1 + k - w.tx0;
            if ((unsigned)a >= (unsigned)w.wx) continue;
            const float p = q.v[1][k];
            const float gx = 0.5f * (q.v[1][k + 1] - q.v[1][k - 1]);
            const float gy = 0.5f * (q.v[2][k] - q.v[0][k]);
            const float so = other_share(A, c, a, b, p);
            f[0] += (double)(p * gx * so);
            f[1] += (double)(p * gy * so);
        }
    }
    cta_fold(f, sh.wf);
    dev::cluster_wait();  // every peer's barriers are initialised
    if (warp == 0) {
        if (lane < kObsBands)
            dev::st_async_v2f64(dev::map_to_rank(dev::smem_addr(&sh.rf[rank][0]), lane), f[0],
                                f[1], dev::map_to_rank(dev::smem_addr(&sh.barF), lane));
        (void)dev::mbar_wait_bounded(&sh.barF, 0, 1u << 24);
        const double Fx = dev::ordered_lane_sum(lane < kObsBands ? sh.rf[lane][0] : 0.0, kObsBands);
        const double Fy = dev::ordered_lane_sum(lane < kObsBands ? sh.rf[lane][1] : 0.0, kObsBands);
        if (lane == 0) {
            const unsigned long long step = *A.step_rd;
            const Words4 r = philox10((uint32_t)(step & 0xFFFFFFFFull), (uint32_t)(step >> 32),
                                      (uint32_t)c.global_id, kTumbleTag,
                                      (uint32_t)(A.polarity_seed & 0xFFFFFFFFull),
                                      (uint32_t)(A.polarity_seed >> 32));
            float theta = c.theta;
            if (u53(r.w[0], r.w[1]) < A.p_tumble) theta = (float)(2.0 * kPi * u53(r.w[2], r.w[3]));
            float sn, co;
            sincosf(theta, &sn, &co);
            sh.vel[0] = (double)c.v_A * (double)co;
            sh.vel[1] = (double)c.v_A * (double)sn;
            sh.vel[2] = (double)A.mot_coeff * Fx;
            sh.vel[3] = (double)A.mot_coeff * Fy;
        }
    }
    __syncthreads();

    // ---- pass 2: centroid-moment channels (FP64 from the binary32 samples)
    const double V = c.V, cx = c.Cx / V, cy = c.Cy / V;
    const double gam = (double)c.gamma, dw = (double)(A.bulk_scale * c.gamma);
    const double vol = (double)(float)(A.vol_scale * (A.A0 - V));
    const double mob = (double)(c.M_pf / (float)kMobilityM0);
    const double rep = (double)A.rep_coeff;
    const double vx = (double)(float)(sh.vel[0] + sh.vel[2]);
    const double vy = (double)(float)(sh.vel[1] + sh.vel[3]);
    double m[8] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    for (int y = y_lo; y < y_hi; y += kObsSweep) {
        const int b = y - w.ty0;
        if ((unsigned)b >= (unsigned)w.wy) continue;
        const Chunk3 q = load_chunk(tile, w, y, ch);
#pragma unroll
        for (int k = 1; k <= 4; ++k) {
            const int a = 4 * ch - 1 + k - w.tx0;
            if ((unsigned)a >= (unsigned)w.wx) continue;
            const double p = q.v[1][k];
            const double e = q.v[1][k + 1], ww = q.v[1][k - 1];
            const double nn = q.v[2][k], s = q.v[0][k];
            const double ne = q.v[2][k + 1], nw = q.v[2][k - 1];
            const double se = q.v[0][k + 1], sw = q.v[0][k - 1];
            const double lap = (4.0 * (nn + s + e + ww) + ne + nw + se + sw - 20.0 * p) / 6.0;
            const double gx = 0.5 * (e - ww), gy = 0.5 * (nn - s);
            const double so = (double)other_share(A, c, a, b, q.v[1][k]);
            double src[4] = {gam * lap - dw * p * (1.0 - p) * (1.0 - 2.0 * p), -rep * p * so,
                             vol * p, -(vx * gx + vy * gy)};
            if (mob != 1.0)  // passive channels only
#pragma unroll
                for (int j = 0; j < 3; ++j) src[j] *= mob;
            const double wx = 2.0 * ((double)a - cx) * p / V;
            const double wy = 2.0 * ((double)b - cy) * p / V;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                m[2 * j] += wx * src[j];
                m[2 * j + 1] += wy * src[j];
            }
        }
    }
    cta_fold(m, sh.wm);
    if (warp != 0) return;
    if (lane == 0) {
        const uint32_t bar = dev::map_to_rank(dev::smem_addr(&sh.barM), 0);
#pragma unroll
        for (int j = 0; j < 8; j += 2)
            dev::st_async_v2f64(dev::map_to_rank(dev::smem_addr(&sh.rm[rank][j]), 0), m[j],
                                m[j + 1], bar);
    }
    if (rank != 0) return;
    if (!dev::mbar_wait_bounded(&sh.barM, 0, 1u << 24)) return;
    double t[8];
#pragma unroll
    for (int j = 0; j < 8; ++j)
        t[j] = dev::ordered_lane_sum(lane < kObsBands ? sh.rm[lane][j] : 0.0, kObsBands);
    if (lane == 0) {
        pfb_moment_accum2d& z = out[n];
        for (int j = 0; j < 4; ++j) z.q[j] += dt * sh.vel[j];
        for (int j = 0; j < 6; ++j) z.q[4 + j] += dt * t[j];
        z.q[10] += dt * (t[6] - sh.vel[0] - sh.vel[2]);
        z.q[11] += dt * (t[7] - sh.vel[1] - sh.vel[3]);
        ++z.count;
    }
}

__global__ void k_zero_advection(pfb_cell2d* cells, int N) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    for (int j = 0; j < 6; ++j) cells[i].advection.q[j] = 0.0;
    cells[i].advection.count = 0ull;
}

}  // namespace

int velocity2d_observe(const pfb_step_args2d& A, pfb_moment_accum2d* out, double dt,
                       cudaStream_t stream) {
    if (!out || !A.cell || !A.phi_in || !A.S_rd || !A.step_rd || A.N < 0 || A.L <= 0)
        return set_error(PFB_E_ARG, "velocity observer: bad arguments");
    if (((uintptr_t)A.phi_in & 15u)) return set_error(PFB_E_ARG, "velocity observer: phi_in must be 16-byte aligned");
    if (A.N == 0) return PFB_OK;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(A.N * kObsBands), 1, 1);
    cfg.blockDim = dim3(kObsThreads, 1, 1);
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = kObsBands;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, k_observe2d, A, out, dt);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return set_error(PFB_E_CUDA, "velocity observer: %s", cudaGetErrorString(e));
    return PFB_OK;
}

// ---- the recorder -----------------------------------------------------------

struct Velocity2D {
    std::string path;
    int stride = 100;
    long long dense = 10000;
    bool reference = false;
    int N = 0;
    double dt = 0.0;
    pfb_moment_accum2d* d_mom = nullptr;
    pfb_moment_accum2d* d_end = nullptr;
    std::vector<pfb_cell2d> cells;
    std::vector<pfb_moment_accum2d> integ, endp;
    std::vector<double> rows;
    std::FILE* f = nullptr;
    long long start = 0, dense_until = 0, last_frame = -1;
    bool primed = false, failed = false;

    ~Velocity2D() {
        if (f) std::fclose(f);
        cudaFree(d_mom);
        cudaFree(d_end);
    }

    bool put(const void* p, size_t n) {
        if (std::fwrite(p, 1, n, f) == n) return true;
        failed = true;
        return false;
    }

    // Host close of the held intervals for a frame (reference
    // common/velocity_moments.h:85-102): e holds dt times the rates the
    // dense observer measures on the current field.
    void finish(pfb_moment_accum2d& m, const pfb_advection_accum& a,
                const pfb_moment_accum2d& e) const {
        m.count = a.count;
        for (int j = 0; j < 4; ++j) m.q[j] = a.q[j];
        if (!m.spatial_count) return;
        const unsigned long long tail = a.count - m.last_sample;
        for (int j = 0; j < 4; ++j) {
            m.q[4 + j] += m.correction[j] + dt * (double)tail * m.held[j];
            const double last = e.q[4 + j] / dt;
            m.q[4 + j] += tail ? dt * 0.5 * (double)(tail - 1) * (last - m.held[j]) : 0.0;
        }
        const double tot[4] = {a.q[0] + a.q[2], a.q[1] + a.q[3], a.q[4], a.q[5]};
        for (int xy = 0; xy < 2; ++xy) {
            const double beta = m.held[4 + xy];
            m.q[10 + xy] += (beta - 1.0) * (tot[xy] - m.last_totals[xy]) +
                            beta * (tot[2 + xy] - m.last_totals[2 + xy]);
        }
    }

    int capture(const pfb_step_args2d& A, long long step, cudaStream_t stream) {
        if (!f || failed || step <= last_frame || A.N != N)
            return set_error(PFB_E_STATE, "velocity recorder: no open file or frame out of order");
        const size_t bytes = (size_t)N * sizeof(pfb_moment_accum2d);
        cudaError_t e = cudaMemsetAsync(d_end, 0, bytes, stream);
        if (e != cudaSuccess) return set_error(PFB_E_CUDA, "velocity: %s", cudaGetErrorString(e));
        int rc = velocity2d_observe(A, d_end, dt, stream);
        if (rc) return rc;
        if ((e = cudaMemcpyAsync(cells.data(), A.cell, (size_t)N * sizeof(pfb_cell2d),
                                 cudaMemcpyDeviceToHost, stream)) != cudaSuccess ||
            (e = cudaMemcpyAsync(integ.data(), d_mom, bytes, cudaMemcpyDeviceToHost, stream)) !=
                cudaSuccess ||
            (e = cudaMemcpyAsync(endp.data(), d_end, bytes, cudaMemcpyDeviceToHost, stream)) !=
                cudaSuccess ||
            (e = cudaStreamSynchronize(stream)) != cudaSuccess)
            return set_error(PFB_E_CUDA, "velocity readback: %s", cudaGetErrorString(e));
        for (int i = 0; i < N; ++i) {
            const pfb_cell2d& c = cells[(size_t)i];
            pfb_moment_accum2d& m = integ[(size_t)i];
            if (!reference) finish(m, c.advection, endp[(size_t)i]);
            if (m.count != (unsigned long long)(step - start)) {
                failed = true;
                return set_error(PFB_E_STATE, "velocity: missed observation at step %lld, cell %d",
                                 step, c.global_id);
            }
            double* row = rows.data() + (size_t)i * kColumns;
            row[0] = c.global_id;
            row[1] = std::fmod((double)c.gx0 + c.Cx / c.V, (double)A.L);
            row[2] = std::fmod((double)c.gy0 + c.Cy / c.V, (double)A.L);
            row[3] = c.theta;
            row[4] = c.gamma;
            row[5] = c.M_pf;
            row[6] = c.v_A;
            row[7] = c.V;
            row[8] = (double)m.count;
            for (int j = 0; j < 12; ++j) row[kIntegralColumn + j] = m.q[j];
            row[kSpatialCountColumn] = (double)(reference ? m.count : m.spatial_count);
            for (int j = 0; j < 4; ++j) row[kEndpointColumn + j] = endp[(size_t)i].q[4 + j] / dt;
            for (int j = 0; j < kColumns; ++j)
                if (!std::isfinite(row[j])) {
                    failed = true;
                    return set_error(PFB_E_STATE, "velocity: non-finite column %d at step %lld, cell %d",
                                     j, step, c.global_id);
                }
        }
        const int64_t disk_step = step;
        if (!put(&disk_step, sizeof(disk_step)) || !put(rows.data(), rows.size() * sizeof(double)) ||
            std::fflush(f) != 0)
            return set_error(PFB_E_IO, "velocity: write failed");
        last_frame = step;
        return PFB_OK;
    }
};

Velocity2D* velocity2d_create(const char* path, int N, double dt, int stride, long long dense,
                              int reference) {
    if (!path || !path[0] || N <= 0 || !std::isfinite(dt) || dt <= 0.0 || stride < 1 ||
        stride > 1000 || dense < 0) {
        set_error(PFB_E_ARG, "velocity recorder: invalid geometry or sampling cadence");
        return nullptr;
    }
    Velocity2D* v = new Velocity2D();
    v->path = path;
    v->N = N;
    v->dt = dt;
    v->stride = stride;
    v->dense = dense;
    v->reference = reference != 0;
    v->cells.resize((size_t)N);
    v->integ.resize((size_t)N);
    v->endp.resize((size_t)N);
    v->rows.resize((size_t)N * kColumns);
    const size_t bytes = (size_t)N * sizeof(pfb_moment_accum2d);
    if (cudaMalloc(&v->d_mom, bytes) != cudaSuccess || cudaMalloc(&v->d_end, bytes) != cudaSuccess ||
        cudaMemset(v->d_mom, 0, bytes) != cudaSuccess) {
        delete v;
        set_error(PFB_E_CUDA, "velocity recorder: allocation failed");
        return nullptr;
    }
    return v;
}

void velocity2d_destroy(Velocity2D* v) { delete v; }

int velocity2d_open(Velocity2D* v, const pfb_step_args2d& A, long long step, cudaStream_t stream) {
    if (v->f || v->failed || step < 0) return set_error(PFB_E_STATE, "velocity recorder already used");
    // a new file only (O_CREAT | O_EXCL)
    v->f = std::fopen(v->path.c_str(), "wbx");
    if (!v->f) {
        v->failed = true;
        return set_error(PFB_E_IO, "velocity: cannot create new output file %s: %s", v->path.c_str(),
                         std::strerror(errno));
    }
    k_zero_advection<<<(v->N + 127) / 128, 128, 0, stream>>>(A.cell, v->N);
    if (cudaGetLastError() != cudaSuccess) return set_error(PFB_E_CUDA, "velocity: zero advection");
    v->start = step;
    const long long dense = v->reference ? 0 : v->dense;
    v->dense_until = step + dense;
    unsigned char h[56] = {};
    std::memcpy(h, "PFVMOM4", 8);
    const uint32_t cells = (uint32_t)v->N, columns = kColumns;
    const double side = (double)A.L;
    const uint32_t stride = v->reference ? 1u : (uint32_t)v->stride, quadrature = 2u;
    const uint64_t dense_u = (uint64_t)dense;
    const int64_t start = step;
    std::memcpy(h + 8, &cells, 4);
    std::memcpy(h + 12, &columns, 4);
    std::memcpy(h + 16, &v->dt, 8);
    std::memcpy(h + 24, &start, 8);
    std::memcpy(h + 32, &side, 8);
    std::memcpy(h + 40, &stride, 4);
    std::memcpy(h + 44, &quadrature, 4);
    std::memcpy(h + 48, &dense_u, 8);
    if (!v->put(h, sizeof(h))) return set_error(PFB_E_IO, "velocity: header write failed");
    return v->capture(A, step, stream);
}

int velocity2d_prepare(Velocity2D* v, pfb_step_args2d* A, long long step, cudaStream_t stream,
                       int* observation) {
    if (v->reference) {
        *observation = PFB_VELOCITY_DISABLED;
        A->moments = nullptr;
        return velocity2d_observe(*A, v->d_mom, v->dt, stream);
    }
    // the reference's graph period is a multiple of the stride, so its slot
    // test (slot % stride) is step % stride
    const bool spatial = !v->primed || step < v->dense_until || step % v->stride == 0;
    *observation = spatial ? PFB_VELOCITY_SPATIAL : PFB_VELOCITY_ADVECTION;
    A->moments = spatial ? v->d_mom : nullptr;
    return PFB_OK;
}

void velocity2d_advanced(Velocity2D* v) { v->primed = true; }

int velocity2d_capture(Velocity2D* v, const pfb_step_args2d& A, long long step,
                       cudaStream_t stream) {
    return v->capture(A, step, stream);
}

long long velocity2d_last_frame(const Velocity2D* v) { return v && v->f ? v->last_frame : -1; }

int velocity2d_close(Velocity2D* v) {
    if (!v->f) return v->failed ? set_error(PFB_E_IO, "velocity recorder failed") : PFB_OK;
    const bool ok = std::fflush(v->f) == 0 && !std::ferror(v->f);
    const bool closed = std::fclose(v->f) == 0;
    v->f = nullptr;
    if (!ok || !closed || v->failed) return set_error(PFB_E_IO, "velocity: close failed");
    return PFB_OK;
}

}  // namespace pfb
