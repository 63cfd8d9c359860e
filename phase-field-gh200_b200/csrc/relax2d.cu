// Relaxation tools around the 2D step, with no counterpart in the reference:
// the step residual r = max over cells and lattice sites of
// |phi_n^{k+1} - phi_n^k| / dt (and its root mean square), and the 64 x 64
// crops that carry a cell between a pfb_sim2d system and the learned
// surrogate (extraction of the network input and of phi targets, insertion of
// a predicted increment).
//
// A cell's window moves on the periodic lattice when it recentres, so both
// use world coordinates: window pixel (i, j) of cell n is lattice site
// ((gx0 + i) mod L, (gy0 + j) mod L) and tile element
// [ty0 + j][tx0 + i] of its 288^2 tile (class window (wx, wy, tx0, ty0)).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <vector>

#include "pfb_common.cuh"
#include "pfb_internal.h"
#include "pfb200_surrogate.h"

namespace pfb {
namespace {

constexpr int kCrop = 64;                 // crop side
constexpr int kCropPad = kCrop + 2;       // padded side of the network input
constexpr int kInCh = 16;                 // network input channels (2 used)
constexpr int kRelaxThreads = 256;

__device__ __forceinline__ int wrap(int v, int L) {
    v %= L;
    return v < 0 ? v + L : v;
}

// phi of cell n at lattice site (x, y), 0 outside its window.
__device__ __forceinline__ float cell_phi_at(const float* tile, const Window& w, int gx0, int gy0,
                                             int x, int y, int L) {
    const int i = wrap(x - gx0, L), j = wrap(y - gy0, L);
    if (i >= w.wx || j >= w.wy) return 0.0f;
    return tile[(size_t)(w.ty0 + j) * kTilePitch + w.tx0 + i];
}

// Residual of the last step: one block per cell, over the union of its new
// and old windows. out[2n] = max |d|, out[2n + 1] = sum d^2 (d = dphi / dt).
__global__ void __launch_bounds__(kRelaxThreads) k_residual2d(
    const float* __restrict__ phi_new, const float* __restrict__ phi_old,
    const pfb_cell2d* __restrict__ c_new, const pfb_cell2d* __restrict__ c_old, int L, double inv_dt,
    double* __restrict__ out) {
    const int n = (int)blockIdx.x;
    const pfb_cell2d a = c_new[n], b = c_old[n];
    const Window wn = window_of(a.cls), wo = window_of(b.cls);
    const float* tn = phi_new + (size_t)n * kTileArea;
    const float* to = phi_old + (size_t)n * kTileArea;
    double mx = 0.0, s2 = 0.0;
    for (int k = (int)threadIdx.x; k < wn.wx * wn.wy; k += kRelaxThreads) {
        const int i = k % wn.wx, j = k / wn.wx;
        const int x = a.gx0 + i, y = a.gy0 + j;
        const float vn = tn[(size_t)(wn.ty0 + j) * kTilePitch + wn.tx0 + i];
        const float vo = cell_phi_at(to, wo, b.gx0, b.gy0, x, y, L);
        const double d = ((double)vn - (double)vo) * inv_dt;
        mx = fmax(mx, fabs(d));
        s2 += d * d;
    }
    // old-window sites outside the new window (new phi there is zero)
    for (int k = (int)threadIdx.x; k < wo.wx * wo.wy; k += kRelaxThreads) {
        const int i = k % wo.wx, j = k / wo.wx;
        const int x = b.gx0 + i, y = b.gy0 + j;
        const int in = wrap(x - a.gx0, L), jn = wrap(y - a.gy0, L);
        if (in < wn.wx && jn < wn.wy) continue;
        const double d = (double)to[(size_t)(wo.ty0 + j) * kTilePitch + wo.tx0 + i] * inv_dt;
        mx = fmax(mx, fabs(d));
        s2 += d * d;
    }
    __shared__ double smx[kRelaxThreads / 32], ss2[kRelaxThreads / 32];
    for (int o = 16; o > 0; o >>= 1) {
        mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, o));
        s2 += __shfl_down_sync(0xffffffffu, s2, o);
    }
    const int w = (int)threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
        smx[w] = mx;
        ss2[w] = s2;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = 0.0, t = 0.0;
        for (int k = 0; k < kRelaxThreads / 32; ++k) {
            m = fmax(m, smx[k]);
            t += ss2[k];
        }
        out[2 * n] = m;
        out[2 * n + 1] = t;
    }
}

// Crop origin of cell n: its centroid rounded, minus half the crop.
__device__ __forceinline__ void crop_origin(const pfb_cell2d& c, int L, int* ox, int* oy) {
    const double V = c.V > 0.0 ? c.V : 1.0;
    const int cx = (int)floor((double)c.gx0 + c.Cx / V + 0.5);
    const int cy = (int)floor((double)c.gy0 + c.Cy / V + 0.5);
    *ox = wrap(cx - kCrop / 2, L);
    *oy = wrap(cy - kCrop / 2, L);
}

// Network input of every cell: a padded 66 x 66 image of 16 bfloat16
// channels, channel 0 = phi_n, channel 1 = sum over the other cells of
// min(phi_m^2, 4) from the exact aggregate (S - q(phi_n)) 2^-27, channel 2 =
// (phi_n - prev) * hist_scale when an earlier crop `prev` at the same origins
// is given (the recent rate of change), else 0; the ring and channels 3..15
// are zero. Origins: the cell's rounded centroid minus half the crop, written
// to `origins`, or read from `origins_in` when given. Also the binary32 phi_n
// crop (optional).
__global__ void __launch_bounds__(kRelaxThreads) k_extract_crops(
    const float* __restrict__ phi, const pfb_cell2d* __restrict__ cells,
    const uint32_t* __restrict__ S, int L, int P, __nv_bfloat16* __restrict__ x0,
    float* __restrict__ phi_crop, int* __restrict__ origins, const int* __restrict__ origins_in,
    const float* __restrict__ prev, float hist_scale) {
    const int n = (int)blockIdx.x;
    const pfb_cell2d c = cells[n];
    const Window w = window_of(c.cls);
    int ox, oy;
    if (origins_in) {
        ox = origins_in[2 * n];
        oy = origins_in[2 * n + 1];
    } else {
        crop_origin(c, L, &ox, &oy);
        if (threadIdx.x == 0) {
            origins[2 * n] = ox;
            origins[2 * n + 1] = oy;
        }
    }
    const float* tile = phi + (size_t)n * kTileArea;
    uint4* img = reinterpret_cast<uint4*>(x0 + (size_t)n * kCropPad * kCropPad * kInCh);
    for (int k = (int)threadIdx.x; k < kCropPad * kCropPad; k += kRelaxThreads) {
        const int u = k % kCropPad - 1, v = k / kCropPad - 1;
        float f = 0.0f, so = 0.0f, rate = 0.0f;
        if (u >= 0 && u < kCrop && v >= 0 && v < kCrop) {
            const int x = wrap(ox + u, L), y = wrap(oy + v, L);
            f = cell_phi_at(tile, w, c.gx0, c.gy0, x, y, L);
            const uint32_t s = S[(size_t)y * P + x];
            const uint32_t q = q_encode(f);
            so = s >= q ? (float)(s - q) * kQInv : 0.0f;
            if (phi_crop) phi_crop[(size_t)n * kCrop * kCrop + v * kCrop + u] = f;
            if (prev) rate = (f - prev[(size_t)n * kCrop * kCrop + v * kCrop + u]) * hist_scale;
        }
        __nv_bfloat162 h01 = __floats2bfloat162_rn(f, so);
        __nv_bfloat162 h23 = __floats2bfloat162_rn(rate, 0.0f);
        uint4 first = make_uint4(*reinterpret_cast<uint32_t*>(&h01), *reinterpret_cast<uint32_t*>(&h23),
                                 0u, 0u);
        img[2 * k] = first;
        img[2 * k + 1] = make_uint4(0u, 0u, 0u, 0u);
    }
}

// out = phi_n crop at the given origins (binary32), minus `minus` if given.
__global__ void __launch_bounds__(kRelaxThreads) k_crop_phi(
    const float* __restrict__ phi, const pfb_cell2d* __restrict__ cells, int L,
    const int* __restrict__ origins, const float* __restrict__ minus, float* __restrict__ out) {
    const int n = (int)blockIdx.x;
    const pfb_cell2d c = cells[n];
    const Window w = window_of(c.cls);
    const int ox = origins[2 * n], oy = origins[2 * n + 1];
    const float* tile = phi + (size_t)n * kTileArea;
    for (int k = (int)threadIdx.x; k < kCrop * kCrop; k += kRelaxThreads) {
        const int u = k % kCrop, v = k / kCrop;
        float f = cell_phi_at(tile, w, c.gx0, c.gy0, wrap(ox + u, L), wrap(oy + v, L), L);
        const size_t o = (size_t)n * kCrop * kCrop + k;
        if (minus) f -= minus[o];
        out[o] = f;
    }
}

// phi_n += dphi at the crop's sites that lie in the cell's window.
__global__ void __launch_bounds__(kRelaxThreads) k_insert_crops(
    float* __restrict__ phi, const pfb_cell2d* __restrict__ cells, int L,
    const int* __restrict__ origins, const float* __restrict__ dphi) {
    const int n = (int)blockIdx.x;
    const pfb_cell2d c = cells[n];
    const Window w = window_of(c.cls);
    const int ox = origins[2 * n], oy = origins[2 * n + 1];
    float* tile = phi + (size_t)n * kTileArea;
    for (int k = (int)threadIdx.x; k < kCrop * kCrop; k += kRelaxThreads) {
        const int u = k % kCrop, v = k / kCrop;
        const int i = wrap(wrap(ox + u, L) - c.gx0, L), j = wrap(wrap(oy + v, L) - c.gy0, L);
        if (i >= w.wx || j >= w.wy) continue;
        tile[(size_t)(w.ty0 + j) * kTilePitch + w.tx0 + i] += dphi[(size_t)n * kCrop * kCrop + k];
    }
}

int need_f32(const Sim2DView& v) {
    if (v.storage != 0) return set_error(PFB_E_CONFIG, "relaxation tools need binary32 pools");
    return PFB_OK;
}

}  // namespace

int relax_extract(pfb_sim2d* s, void* x0, float* phi_crop, int* origins, const int* origins_in,
                  const float* prev, float hist_scale) {
    Sim2DView v;
    int rc = sim2d_view(s, &v);
    if (rc || (rc = need_f32(v))) return rc;
    if (!x0 || (!origins && !origins_in)) return set_error(PFB_E_ARG, "extract: null buffer");
    cudaSetDevice(v.device);
    k_extract_crops<<<v.N, kRelaxThreads, 0, v.stream>>>(v.phi_cur, v.cells, v.S_cur, v.L, v.P,
                                                        static_cast<__nv_bfloat16*>(x0), phi_crop,
                                                        origins, origins_in, prev, hist_scale);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? PFB_OK : set_error(PFB_E_CUDA, "extract: %s", cudaGetErrorString(e));
}

int relax_insert(pfb_sim2d* s, const int* origins, const float* dphi) {
    Sim2DView v;
    int rc = sim2d_view(s, &v);
    if (rc || (rc = need_f32(v))) return rc;
    if (!origins || !dphi) return set_error(PFB_E_ARG, "insert: null buffer");
    cudaSetDevice(v.device);
    k_insert_crops<<<v.N, kRelaxThreads, 0, v.stream>>>(v.phi_cur, v.cells, v.L, origins, dphi);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return set_error(PFB_E_CUDA, "insert: %s", cudaGetErrorString(e));
    return sim2d_rebuild(s);
}

}  // namespace pfb

using namespace pfb;

extern "C" {

int pfb_sim2d_residual_step(pfb_sim2d* s, double* linf, double* rms) {
    clear_error();
    Sim2DView v;
    int rc = sim2d_view(s, &v);
    if (rc || (rc = need_f32(v))) return rc;
    if (cudaSetDevice(v.device) != cudaSuccess) return set_error(PFB_E_CUDA, "cudaSetDevice");
    rc = sim2d_step_keep_prev(s);
    if (rc) return rc;
    rc = sim2d_view(s, &v);
    if (rc) return rc;
    double* d_out = nullptr;
    cudaError_t e = cudaMallocAsync(&d_out, (size_t)v.N * 2 * sizeof(double), v.stream);
    if (e != cudaSuccess) return set_error(PFB_E_CUDA, "residual alloc: %s", cudaGetErrorString(e));
    k_residual2d<<<v.N, kRelaxThreads, 0, v.stream>>>(v.phi_cur, v.phi_prev, v.cells, v.cells_prev,
                                                       v.L, 1.0 / v.dt, d_out);
    std::vector<double> h((size_t)v.N * 2);
    e = cudaMemcpyAsync(h.data(), d_out, h.size() * sizeof(double), cudaMemcpyDeviceToHost, v.stream);
    cudaFreeAsync(d_out, v.stream);
    const cudaError_t e2 = cudaStreamSynchronize(v.stream);
    if (e != cudaSuccess || e2 != cudaSuccess)
        return set_error(PFB_E_CUDA, "residual: %s", cudaGetErrorString(e != cudaSuccess ? e : e2));
    double mx = 0.0, s2 = 0.0, area = 0.0;
    std::vector<pfb_cell2d> cells((size_t)v.N);
    e = cudaMemcpy(cells.data(), v.cells, cells.size() * sizeof(pfb_cell2d), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return set_error(PFB_E_CUDA, "residual: %s", cudaGetErrorString(e));
    for (int n = 0; n < v.N; ++n) {
        mx = std::fmax(mx, h[(size_t)2 * n]);
        s2 += h[(size_t)2 * n + 1];
        const Window w = window_of(cells[(size_t)n].cls);
        area += (double)w.wx * w.wy;
    }
    if (linf) *linf = mx;
    if (rms) *rms = std::sqrt(s2 / area);
    return PFB_OK;
}

int pfb_sur2d_extract(pfb_sim2d* s, void* x0, float* phi_crop, int* origins) {
    clear_error();
    return relax_extract(s, x0, phi_crop, origins, nullptr, nullptr, 0.0f);
}

int pfb_sur2d_extract_at(pfb_sim2d* s, const int* origins, const float* prev, float hist_scale,
                         void* x0, float* phi_crop) {
    clear_error();
    if (!origins) return set_error(PFB_E_ARG, "extract_at: null origins");
    return relax_extract(s, x0, phi_crop, nullptr, origins, prev, hist_scale);
}

int pfb_sur2d_crop_phi(pfb_sim2d* s, const int* origins, const float* minus, float* out) {
    clear_error();
    Sim2DView v;
    int rc = sim2d_view(s, &v);
    if (rc || (rc = need_f32(v))) return rc;
    if (!origins || !out) return set_error(PFB_E_ARG, "crop_phi: null buffer");
    cudaSetDevice(v.device);
    k_crop_phi<<<v.N, kRelaxThreads, 0, v.stream>>>(v.phi_cur, v.cells, v.L, origins, minus, out);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? PFB_OK : set_error(PFB_E_CUDA, "crop_phi: %s", cudaGetErrorString(e));
}

int pfb_sur2d_insert(pfb_sim2d* s, const int* origins, const float* dphi) {
    clear_error();
    return relax_insert(s, origins, dphi);
}

}  // extern "C"
