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

constexpr int kObsThreads = 256;
constexpr int kObsWarps = kObsThreads / 32;
constexpr int kColumns = 26;        // PFVMOM4 columns per cell
constexpr int kIntegralColumn = 9;  // q[0..11]
constexpr int kSpatialCountColumn = 21;
constexpr int kEndpointColumn = 22;

__device__ __forceinline__ float tile_at(const float* tile, const Window& w, int x, int y) {
    if ((unsigned)x >= (unsigned)w.wx || (unsigned)y >= (unsigned)w.wy) return 0.0f;
    return tile[(w.ty0 + y) * kTilePitch + w.tx0 + x];
}

// S_other at window pixel (x, y); an aggregate below the cell's own share is
// returned as NaN so that a frame built from it is refused.
__device__ __forceinline__ float other_at(const pfb_step_args2d& A, const pfb_cell2d& c, int x,
                                          int y, float p) {
    const int gx = (c.gx0 + x) % A.L, gy = (c.gy0 + y) % A.L;
    const uint32_t all = A.S_rd[(size_t)gy * A.P + gx], self = q_encode(p);
    return all >= self ? (float)(all - self) * kQInv : __int_as_float(0x7fc00000);
}

// Block sum of NV doubles: warp shuffles, then ascending warps by thread 0;
// the totals land in red[j][0].
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double (*red)[kObsWarps]) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int j = 0; j < NV; ++j) {
        const double s = dev::warp_sum_down(v[j]);
        if (lane == 0) red[j][warp] = s;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int j = 0; j < NV; ++j) {
            double s = 0.0;
            for (int w = 0; w < kObsWarps; ++w) s += red[j][w];
            red[j][0] = s;
        }
    }
    __syncthreads();
}

// One CTA per cell: the velocity the step would take (tumble included) and
// the twelve centroid-moment channels of phi^n, each rate times dt added to
// out[n] (reference src/velocity_moments.cu:47-123).
__global__ void __launch_bounds__(kObsThreads)
    k_observe2d(const __grid_constant__ pfb_step_args2d A, pfb_moment_accum2d* out, double dt) {
    const int n = blockIdx.x, tid = threadIdx.x;
    const pfb_cell2d& c = A.cell[n];
    const Window w = window_of(c.cls);
    const float* tile = A.phi_in + (size_t)n * kTileArea;
    __shared__ double red[8][kObsWarps];
    __shared__ double vel[4];
    const int area = w.wx * w.wy;

    double f[2] = {0.0, 0.0};
    for (int k = tid; k < area; k += kObsThreads) {
        const int x = k % w.wx, y = k / w.wx;
        const float p = tile_at(tile, w, x, y);
        const float gx = 0.5f * (tile_at(tile, w, x + 1, y) - tile_at(tile, w, x - 1, y));
        const float gy = 0.5f * (tile_at(tile, w, x, y + 1) - tile_at(tile, w, x, y - 1));
        const float so = other_at(A, c, x, y, p);
        f[0] += (double)(p * gx * so);
        f[1] += (double)(p * gy * so);
    }
    block_sum(f, red);
    if (tid == 0) {
        const unsigned long long step = *A.step_rd;
        const Words4 r = philox10((uint32_t)(step & 0xFFFFFFFFull), (uint32_t)(step >> 32),
                                  (uint32_t)c.global_id, kTumbleTag,
                                  (uint32_t)(A.polarity_seed & 0xFFFFFFFFull),
                                  (uint32_t)(A.polarity_seed >> 32));
        float theta = c.theta;
        if (u53(r.w[0], r.w[1]) < A.p_tumble) theta = (float)(2.0 * kPi * u53(r.w[2], r.w[3]));
        float sn, co;
        sincosf(theta, &sn, &co);
        vel[0] = (double)c.v_A * (double)co;
        vel[1] = (double)c.v_A * (double)sn;
        vel[2] = (double)A.mot_coeff * red[0][0];
        vel[3] = (double)A.mot_coeff * red[1][0];
    }
    __syncthreads();
    const double cx = c.Cx / c.V, cy = c.Cy / c.V;
    const double dw = (double)(A.bulk_scale * c.gamma);
    const double vol = (double)(float)(A.vol_scale * (A.A0 - c.V));
    const double mobility = (double)(c.M_pf / (float)kMobilityM0);
    const double vx = (double)(float)(vel[0] + vel[2]);
    const double vy = (double)(float)(vel[1] + vel[3]);
    double m[8] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    for (int k = tid; k < area; k += kObsThreads) {
        const int x = k % w.wx, y = k / w.wx;
        const double p = tile_at(tile, w, x, y);
        const double e = tile_at(tile, w, x + 1, y), ww = tile_at(tile, w, x - 1, y);
        const double nn = tile_at(tile, w, x, y + 1), s = tile_at(tile, w, x, y - 1);
        const double ne = tile_at(tile, w, x + 1, y + 1), nw = tile_at(tile, w, x - 1, y + 1);
        const double se = tile_at(tile, w, x + 1, y - 1), sw = tile_at(tile, w, x - 1, y - 1);
        const double lap = (4.0 * (nn + s + e + ww) + ne + nw + se + sw - 20.0 * p) / 6.0;
        const double gx = 0.5 * (e - ww), gy = 0.5 * (nn - s);
        const double so = (double)other_at(A, c, x, y, (float)p);
        double src[4] = {(double)c.gamma * lap - dw * p * (1.0 - p) * (1.0 - 2.0 * p),
                         -(double)A.rep_coeff * p * so, vol * p, -(vx * gx + vy * gy)};
        // the mobility scales the passive terms, never advection
        if (mobility != 1.0)
            for (int j = 0; j < 3; ++j) src[j] *= mobility;
        const double wx = 2.0 * ((double)x - cx) * p / c.V;
        const double wy = 2.0 * ((double)y - cy) * p / c.V;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            m[2 * j] += wx * src[j];
            m[2 * j + 1] += wy * src[j];
        }
    }
    block_sum(m, red);
    if (tid == 0) {
        pfb_moment_accum2d& z = out[n];
        for (int j = 0; j < 4; ++j) z.q[j] += dt * vel[j];
        for (int j = 0; j < 6; ++j) z.q[4 + j] += dt * red[j][0];
        z.q[10] += dt * (red[6][0] - vel[0] - vel[2]);
        z.q[11] += dt * (red[7][0] - vel[1] - vel[3]);
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
    if (A.N == 0) return PFB_OK;
    k_observe2d<<<A.N, kObsThreads, 0, stream>>>(A, out, dt);
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
