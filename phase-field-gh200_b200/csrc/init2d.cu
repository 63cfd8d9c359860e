// Initialisation and diagnostic kernels of the 2D path: tanh-disk seeding,
// initial moments, the S rebuild from a phi pool, verification and the
// trajectory pack (reference src/kernels.cu:1044-1265; behaviour restated).
#include <cuda_runtime.h>

#include <cstdint>

#include "device_util.cuh"
#include "pfb_common.cuh"
#include "pfb_internal.h"
#include "storage2d.cuh"

#include <algorithm>

namespace pfb {

namespace {

__device__ __forceinline__ int wrap_side(int v, int L) {
    v %= L;
    return v < 0 ? v + L : v;
}

// Zero both tiles of cell n, then seed phi = (1 - tanh(k (r - R_eff)))/2 in
// the class window of pool a, centred on the periodic image nearest (cx, cy).
__global__ void k_init_tiles2d(float* phi_a, float* phi_b, pfb_cell2d* cell, const uint8_t* clsv,
                               int N, int L, const float* seed_cx, const float* seed_cy,
                               float radius_eff, float kappa_iface) {
    const int n = blockIdx.x;
    if (n >= N) return;
    const int cls = (int)clsv[n];
    const Window w = window_of(cls);
    float* ta = phi_a + (size_t)n * kTileArea;
    float* tb = phi_b + (size_t)n * kTileArea;
    for (int i = threadIdx.x; i < kTileArea; i += blockDim.x) {
        ta[i] = 0.0f;
        tb[i] = 0.0f;
    }
    __syncthreads();
    const float cx = seed_cx[n], cy = seed_cy[n];
    const int gx0 = wrap_side((int)lrintf(cx - 0.5f * (float)(w.wx - 1)), L);
    const int gy0 = wrap_side((int)lrintf(cy - 0.5f * (float)(w.wy - 1)), L);
    const float half = 0.5f * (float)L;
    for (int p = threadIdx.x; p < w.wx * w.wy; p += blockDim.x) {
        const int a = p % w.wx, b = p / w.wx;
        float dx = (float)(gx0 + a) - cx;
        float dy = (float)(gy0 + b) - cy;
        if (dx > half) dx -= (float)L;
        if (dx < -half) dx += (float)L;
        if (dy > half) dy -= (float)L;
        if (dy < -half) dy += (float)L;
        const float r = sqrtf(dx * dx + dy * dy);
        ta[(size_t)(w.ty0 + b) * kTilePitch + w.tx0 + a] =
            0.5f * (1.0f - tanhf(kappa_iface * (r - radius_eff)));
    }
    if (threadIdx.x == 0) {
        pfb_cell2d& cs = cell[n];
        cs.gx0 = gx0;
        cs.gy0 = gy0;
        cs.cls = (uint8_t)cls;
        cs.cls_written[0] = (uint8_t)cls;
        cs.cls_written[1] = (uint8_t)cls;
    }
}

// V, Cx, Cy, support box, phi_max of the class window; clears the demotion
// counter and the interaction integral.
__global__ void __launch_bounds__(256) k_init_moments2d(pfb_cell2d* cell, const uint8_t* clsv,
                                                        const float* phi, int N) {
    __shared__ double sd[8][3];
    __shared__ int si[8][5];
    const int n = blockIdx.x;
    if (n >= N) return;
    const Window w = window_of((int)clsv[n]);
    const float* t = phi + (size_t)n * kTileArea;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double aV = 0.0, aCx = 0.0, aCy = 0.0;
    int blox = w.wx, bhix = -1, bloy = w.wy, bhiy = -1, pmaxb = 0;
    for (int b = warp; b < w.wy; b += 8) {
        for (int a = lane; a < w.wx; a += 32) {
            const float pn = t[(size_t)(w.ty0 + b) * kTilePitch + w.tx0 + a];
            const double d = (double)pn * (double)pn;
            aV += d;
            aCx += d * (double)a;
            aCy += d * (double)b;
            pmaxb = max(pmaxb, (int)__float_as_uint(fabsf(pn)));
            if (pn > kSupportEps) {
                blox = min(blox, a);
                bhix = max(bhix, a);
                bloy = min(bloy, b);
                bhiy = max(bhiy, b);
            }
        }
    }
    aV = dev::warp_sum_down(aV);
    aCx = dev::warp_sum_down(aCx);
    aCy = dev::warp_sum_down(aCy);
    blox = dev::warp_min_down(blox);
    bhix = dev::warp_max_down(bhix);
    bloy = dev::warp_min_down(bloy);
    bhiy = dev::warp_max_down(bhiy);
    pmaxb = dev::warp_max_down(pmaxb);
    if (lane == 0) {
        sd[warp][0] = aV;
        sd[warp][1] = aCx;
        sd[warp][2] = aCy;
        si[warp][0] = blox;
        si[warp][1] = bhix;
        si[warp][2] = bloy;
        si[warp][3] = bhiy;
        si[warp][4] = pmaxb;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double m[3] = {0.0, 0.0, 0.0};
        int bb[5] = {w.wx, -1, w.wy, -1, 0};
        for (int k = 0; k < 8; ++k) {
            m[0] += sd[k][0];
            m[1] += sd[k][1];
            m[2] += sd[k][2];
            bb[0] = min(bb[0], si[k][0]);
            bb[1] = max(bb[1], si[k][1]);
            bb[2] = min(bb[2], si[k][2]);
            bb[3] = max(bb[3], si[k][3]);
            bb[4] = max(bb[4], si[k][4]);
        }
        pfb_cell2d& cs = cell[n];
        cs.V = m[0];
        cs.Cx = m[1];
        cs.Cy = m[2];
        cs.bb_lo_x = bb[0];
        cs.bb_hi_x = bb[1];
        cs.bb_lo_y = bb[2];
        cs.bb_hi_y = bb[3];
        cs.phi_max = __uint_as_float((uint32_t)bb[4]);
        cs.promote_ctr = 0u;
        cs.Ix = 0.0;
        cs.Iy = 0.0;
    }
}

__global__ void k_scatter_all2d(const float* phi, const pfb_cell2d* cell, const uint8_t* clsv,
                                uint32_t* S, int N, int L, int P, uint32_t* flags) {
    const int n = blockIdx.x;
    if (n >= N) return;
    const Window w = window_of((int)clsv[n]);
    const int gx0 = cell[n].gx0, gy0 = cell[n].gy0;
    const float* t = phi + (size_t)n * kTileArea;
    for (int p = threadIdx.x; p < w.wx * w.wy; p += blockDim.x) {
        const int a = p % w.wx, b = p / w.wx;
        const float pn = t[(size_t)(w.ty0 + b) * kTilePitch + w.tx0 + a];
        const uint32_t q = q_encode(pn);
        if (!q) continue;
        const int gx = wrap_side(gx0 + a, L);
        const int gy = wrap_side(gy0 + b, L);
        const uint32_t old = atomicAdd(S + (size_t)gy * P + gx, q);
        if (old > 0xFFFFFFFFu - q) atomicOr(flags + PFB_FLAG_S_OVERFLOW, 1u);
        if (pn * pn > kPhiSqCap) atomicOr(flags + PFB_FLAG_Q_CLAMP, 1u);
    }
}

__global__ void k_zero_u32(uint32_t* p, size_t n) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x)
        p[i] = 0u;
}

__global__ void __launch_bounds__(256) k_verify_cells2d(const float* phi, const pfb_cell2d* cell,
                                                        const uint8_t* clsv, int N, double* out_V,
                                                        float* out_outside) {
    __shared__ double sv[8];
    __shared__ float so[8];
    const int n = blockIdx.x;
    if (n >= N) return;
    const Window w = window_of((int)clsv[n]);
    const float* t = phi + (size_t)n * kTileArea;
    double v = 0.0;
    float omax = 0.0f;
    for (int i = threadIdx.x; i < kTileArea; i += blockDim.x) {
        const int x = i % kTilePitch, y = i / kTilePitch;
        const float p = t[i];
        const bool inside = x >= w.tx0 && x < w.tx0 + w.wx && y >= w.ty0 && y < w.ty0 + w.wy;
        if (inside)
            v += (double)p * (double)p;
        else
            omax = fmaxf(omax, fabsf(p));
    }
    v = dev::warp_sum_down(v);
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) omax = fmaxf(omax, __shfl_down_sync(0xFFFFFFFFu, omax, d));
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
        sv[warp] = v;
        so[warp] = omax;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        float o = 0.0f;
        for (int k = 0; k < 8; ++k) {
            s += sv[k];
            o = fmaxf(o, so[k]);
        }
        out_V[n] = s;
        out_outside[n] = o;
    }
}

__global__ void k_verify_S(const uint32_t* S, size_t n, uint32_t* out_max) {
    uint32_t m = 0u;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x)
        m = max(m, S[i]);
    atomicMax(out_max, m);
}

__global__ void k_pack_traj2d(const pfb_cell2d* cell, const uint8_t* clsv, pfb_traj_cell2d* out,
                              int N, int L) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    const pfb_cell2d& cs = cell[n];
    const double V = cs.V > 0.0 ? cs.V : 1.0;
    const double cx = (double)cs.gx0 + cs.Cx / V;
    const double cy = (double)cs.gy0 + cs.Cy / V;
    pfb_traj_cell2d t;
    t.global_id = cs.global_id;
    t.cls = (int32_t)clsv[n];
    t.cx = (float)(cx - floor(cx / (double)L) * (double)L);
    t.cy = (float)(cy - floor(cy / (double)L) * (double)L);
    t.vx = cs.vx;
    t.vy = cs.vy;
    t.theta = cs.theta;
    t.volume = (float)cs.V;
    t.perim = (float)cs.perim;
    t.gamma = cs.gamma;
    t.v_A = cs.v_A;
    t.phi_max = cs.phi_max;
    out[n] = t;
}

int launch_status(const char* what) {
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return set_error(PFB_E_CUDA, "%s: %s", what, cudaGetErrorString(e));
    return PFB_OK;
}

}  // namespace

int init_tiles2d(float* phi_a, float* phi_b, pfb_cell2d* cell, const uint8_t* cls, int N, int L,
                 const float* cx, const float* cy, float radius_eff, float kappa_iface,
                 cudaStream_t s) {
    if (!phi_a || !phi_b || !cell || !cls || !cx || !cy || N < 0 || L <= 0)
        return set_error(PFB_E_ARG, "init_tiles2d: bad argument");
    if (N == 0) return PFB_OK;
    k_init_tiles2d<<<N, 256, 0, s>>>(phi_a, phi_b, cell, cls, N, L, cx, cy, radius_eff,
                                      kappa_iface);
    return launch_status("init_tiles2d");
}

int init_moments2d(pfb_cell2d* cell, const uint8_t* cls, const float* phi, int N, cudaStream_t s) {
    if (!cell || !cls || !phi || N < 0) return set_error(PFB_E_ARG, "init_moments2d: bad argument");
    if (N == 0) return PFB_OK;
    k_init_moments2d<<<N, 256, 0, s>>>(cell, cls, phi, N);
    return launch_status("init_moments2d");
}

int scatter_all2d(const float* phi, const pfb_cell2d* cell, const uint8_t* cls, uint32_t* S,
                  int N, int L, int P, uint32_t* flags, cudaStream_t s) {
    if (!phi || !cell || !cls || !S || !flags || N < 0 || L <= 0 || P < L)
        return set_error(PFB_E_ARG, "scatter_all2d: bad argument");
    if (N == 0) return PFB_OK;
    k_scatter_all2d<<<N, 256, 0, s>>>(phi, cell, cls, S, N, L, P, flags);
    return launch_status("scatter_all2d");
}

int zero_u32(uint32_t* p, size_t n, cudaStream_t s) {
    if (!p && n) return set_error(PFB_E_ARG, "zero_u32: null");
    if (!n) return PFB_OK;
    size_t blocks = (n + 255) / 256;
    if (blocks > 4096) blocks = 4096;
    k_zero_u32<<<(unsigned)blocks, 256, 0, s>>>(p, n);
    return launch_status("zero_u32");
}

int verify_cells2d(const float* phi, const pfb_cell2d* cell, const uint8_t* cls, int N,
                   double* out_V, float* out_outside, cudaStream_t s) {
    if (!phi || !cell || !cls || !out_V || !out_outside || N < 0)
        return set_error(PFB_E_ARG, "verify_cells2d: bad argument");
    if (N == 0) return PFB_OK;
    k_verify_cells2d<<<N, 256, 0, s>>>(phi, cell, cls, N, out_V, out_outside);
    return launch_status("verify_cells2d");
}

int verify_S(const uint32_t* S, size_t n, uint32_t* out_max, cudaStream_t s) {
    if (!S || !out_max) return set_error(PFB_E_ARG, "verify_S: null");
    if (!n) return PFB_OK;
    k_verify_S<<<256, 256, 0, s>>>(S, n, out_max);
    return launch_status("verify_S");
}

int pack_traj2d(const pfb_cell2d* cell, const uint8_t* cls, pfb_traj_cell2d* out, int N, int L,
                cudaStream_t s) {
    if (!cell || !cls || !out || N < 0 || L <= 0) return set_error(PFB_E_ARG, "pack_traj2d: bad argument");
    if (N == 0) return PFB_OK;
    k_pack_traj2d<<<(N + 127) / 128, 128, 0, s>>>(cell, cls, out, N, L);
    return launch_status("pack_traj2d");
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
