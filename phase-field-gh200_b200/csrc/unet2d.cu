// The learned relaxation surrogate: a small U-Net on 64 x 64 crops, built
// from the tcgen05 convolutions of conv2d_tc.cu, with its training step
// (mean-squared error, Adam) and the jump of a pfb_sim2d system. No
// counterpart in the reference.
//
// Input: 3 channels (phi_n, the other cells' sum of phi^2 and phi_n's recent
// rate of change, padded to 16).
// Output: the increment of phi_n over a fixed number of passive relaxation
// steps (channel 0 of 16). Layers (3x3, width 32, ReLU except the last):
//   c1 16->32 @64, c2 32->32 @64 (skip), 2x2 average pool,
//   c3 32->32 @32, c4 32->32 @32, nearest upsample + skip,
//   c5, c6, c7 32->32 @64, c8 32->16 @64 (linear).
// Activations are bfloat16 in the padded channels-last layout; every
// contraction accumulates in binary32 in TMEM; master weights, gradients and
// Adam moments are binary32. The data gradient of a layer is its forward
// kernel run with flipped, transposed weights, with the ReLU derivative of
// the layer below fused as a gate.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "pfb_internal.h"
#include "pfb200_surrogate.h"

using namespace pfb;

namespace {

using bf16 = __nv_bfloat16;

constexpr int kImg = 64, kHalf = 32;
constexpr int kP64 = (kImg + 2) * (kImg + 2), kP32 = (kHalf + 2) * (kHalf + 2);
constexpr int kEwThreads = 256;

struct LayerSpec {
    int cin, cout, res, relu, cin_real, cout_real;
};
constexpr LayerSpec kLayers[8] = {{16, 32, 64, 1, 3, 32},  {32, 32, 64, 1, 32, 32},
                                  {32, 32, 32, 1, 32, 32}, {32, 32, 32, 1, 32, 32},
                                  {32, 32, 64, 1, 32, 32}, {32, 32, 64, 1, 32, 32},
                                  {32, 32, 64, 1, 32, 32}, {32, 16, 64, 0, 32, 1}};

__device__ __forceinline__ int q64(int y, int x) { return (y + 1) * (kImg + 2) + x + 1; }
__device__ __forceinline__ int q32(int y, int x) { return (y + 1) * (kHalf + 2) + x + 1; }

__device__ __forceinline__ void unpack8(const uint4& v, float* f) {
    const __nv_bfloat162* h = reinterpret_cast<const __nv_bfloat162*>(&v);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const float2 t = __bfloat1622float2(h[j]);
        f[2 * j] = t.x;
        f[2 * j + 1] = t.y;
    }
}
__device__ __forceinline__ uint4 pack8(const float* f) {
    uint4 v;
    __nv_bfloat162* h = reinterpret_cast<__nv_bfloat162*>(&v);
#pragma unroll
    for (int j = 0; j < 4; ++j) h[j] = __floats2bfloat162_rn(f[2 * j], f[2 * j + 1]);
    return v;
}

// 32-channel tensors are handled as 4 vectors of 8 channels per position.
__global__ void k_pool2(const uint4* __restrict__ a, uint4* __restrict__ p, int B) {
    const int n = B * kHalf * kHalf * 4;
    for (int t = (int)(blockIdx.x * blockDim.x + threadIdx.x); t < n; t += gridDim.x * blockDim.x) {
        const int c4 = t & 3, pix = t >> 2;
        const int b = pix / (kHalf * kHalf), r = pix - b * kHalf * kHalf;
        const int i = r / kHalf, j = r - (r / kHalf) * kHalf;
        const uint4* ab = a + (size_t)b * kP64 * 4;
        float s[8] = {}, f[8];
#pragma unroll
        for (int d = 0; d < 4; ++d) {
            unpack8(ab[q64(2 * i + (d >> 1), 2 * j + (d & 1)) * 4 + c4], f);
#pragma unroll
            for (int k = 0; k < 8; ++k) s[k] += f[k];
        }
#pragma unroll
        for (int k = 0; k < 8; ++k) s[k] *= 0.25f;
        p[((size_t)b * kP32 + q32(i, j)) * 4 + c4] = pack8(s);
    }
}

__global__ void k_upadd(const uint4* __restrict__ a32, const uint4* __restrict__ skip,
                        uint4* __restrict__ u, int B) {
    const int n = B * kImg * kImg * 4;
    for (int t = (int)(blockIdx.x * blockDim.x + threadIdx.x); t < n; t += gridDim.x * blockDim.x) {
        const int c4 = t & 3, pix = t >> 2;
        const int b = pix / (kImg * kImg), r = pix - b * kImg * kImg;
        const int y = r / kImg, x = r - (r / kImg) * kImg;
        float f[8], g[8];
        unpack8(a32[((size_t)b * kP32 + q32(y >> 1, x >> 1)) * 4 + c4], f);
        const size_t o = ((size_t)b * kP64 + q64(y, x)) * 4 + c4;
        unpack8(skip[o], g);
#pragma unroll
        for (int k = 0; k < 8; ++k) f[k] += g[k];
        u[o] = pack8(f);
    }
}

// dz4 = (sum of the 2x2 upsampling gradient) * (a4 > 0)
__global__ void k_upback_gate(const uint4* __restrict__ gu, const uint4* __restrict__ a4,
                              uint4* __restrict__ dz4, int B) {
    const int n = B * kHalf * kHalf * 4;
    for (int t = (int)(blockIdx.x * blockDim.x + threadIdx.x); t < n; t += gridDim.x * blockDim.x) {
        const int c4 = t & 3, pix = t >> 2;
        const int b = pix / (kHalf * kHalf), r = pix - b * kHalf * kHalf;
        const int i = r / kHalf, j = r - (r / kHalf) * kHalf;
        float s[8] = {}, f[8], g[8];
#pragma unroll
        for (int d = 0; d < 4; ++d) {
            unpack8(gu[((size_t)b * kP64 + q64(2 * i + (d >> 1), 2 * j + (d & 1))) * 4 + c4], f);
#pragma unroll
            for (int k = 0; k < 8; ++k) s[k] += f[k];
        }
        const size_t o = ((size_t)b * kP32 + q32(i, j)) * 4 + c4;
        unpack8(a4[o], g);
#pragma unroll
        for (int k = 0; k < 8; ++k) s[k] = g[k] > 0.0f ? s[k] : 0.0f;
        dz4[o] = pack8(s);
    }
}

// dz2 = (pool gradient gp / 4 broadcast + skip gradient gu) * (a2 > 0)
__global__ void k_skipgrad(const uint4* __restrict__ gp, const uint4* __restrict__ gu,
                           const uint4* __restrict__ a2, uint4* __restrict__ dz2, int B) {
    const int n = B * kImg * kImg * 4;
    for (int t = (int)(blockIdx.x * blockDim.x + threadIdx.x); t < n; t += gridDim.x * blockDim.x) {
        const int c4 = t & 3, pix = t >> 2;
        const int b = pix / (kImg * kImg), r = pix - b * kImg * kImg;
        const int y = r / kImg, x = r - (r / kImg) * kImg;
        float f[8], g[8], a[8];
        unpack8(gp[((size_t)b * kP32 + q32(y >> 1, x >> 1)) * 4 + c4], f);
        const size_t o = ((size_t)b * kP64 + q64(y, x)) * 4 + c4;
        unpack8(gu[o], g);
        unpack8(a2[o], a);
#pragma unroll
        for (int k = 0; k < 8; ++k) f[k] = a[k] > 0.0f ? 0.25f * f[k] + g[k] : 0.0f;
        dz2[o] = pack8(f);
    }
}

// Mean-squared error of channel 0 of the output against the target
// increment; writes the output gradient (16 channels, channel 0 used) and one
// partial sum of squares per block (fixed grid, summed in order on the host).
constexpr int kLossBlocks = 256;
__global__ void __launch_bounds__(kEwThreads) k_loss(const float* __restrict__ out,
                                                     const float* __restrict__ target,
                                                     uint4* __restrict__ go, double* __restrict__ partial,
                                                     int B, float scale) {
    const int n = B * kImg * kImg;
    double s = 0.0;
    for (int t = (int)(blockIdx.x * blockDim.x + threadIdx.x); t < n; t += gridDim.x * blockDim.x) {
        const int b = t / (kImg * kImg), r = t - b * kImg * kImg;
        const int q = q64(r / kImg, r % kImg);
        const float d = out[((size_t)b * kP64 + q) * 16] - target[t];
        s += (double)d * d;
        const float g = 2.0f * d * scale;
        __nv_bfloat162 h = __floats2bfloat162_rn(g, 0.0f);
        const size_t o = ((size_t)b * kP64 + q) * 2;
        go[o] = make_uint4(*reinterpret_cast<uint32_t*>(&h), 0u, 0u, 0u);
        go[o + 1] = make_uint4(0u, 0u, 0u, 0u);
    }
    __shared__ double red[kEwThreads / 32];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int k = 0; k < kEwThreads / 32; ++k) t += red[k];
        partial[blockIdx.x] = t;
    }
}

__global__ void k_adam(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, long long n, float lr, float b1, float b2, float eps,
                       float bc1, float bc2) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.0f - b1) * gi;
        const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        p[i] -= lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
    }
}

// Batch assembly: images idx[k] of the training set into slot k.
__global__ void k_gather(const uint4* __restrict__ x_all, const float* __restrict__ t_all,
                         const int* __restrict__ idx, uint4* __restrict__ x0, float* __restrict__ t) {
    const int k = (int)blockIdx.x;
    const size_t src = (size_t)idx[k];
    for (int i = (int)threadIdx.x; i < kP64 * 2; i += blockDim.x)
        x0[(size_t)k * kP64 * 2 + i] = x_all[src * kP64 * 2 + i];
    for (int i = (int)threadIdx.x; i < kImg * kImg; i += blockDim.x)
        t[(size_t)k * kImg * kImg + i] = t_all[src * kImg * kImg + i];
}

__global__ void k_take_ch0(const float* __restrict__ out, float* __restrict__ d, int B) {
    const int n = B * kImg * kImg;
    for (int t = (int)(blockIdx.x * blockDim.x + threadIdx.x); t < n; t += gridDim.x * blockDim.x) {
        const int b = t / (kImg * kImg), r = t - b * kImg * kImg;
        d[t] = out[((size_t)b * kP64 + q64(r / kImg, r % kImg)) * 16];
    }
}

int ew_blocks(long long n) {
    const long long b = (n + kEwThreads - 1) / kEwThreads;
    return (int)(b < 148 * 16 ? b : 148 * 16);
}

// splitmix64-driven Box-Muller normal deviates (reproducible across hosts).
struct Rng {
    unsigned long long s;
    unsigned long long next() {
        unsigned long long z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    double uniform() { return ((next() >> 11) + 0.5) * (1.0 / 9007199254740992.0); }
    double normal() {
        const double u1 = uniform(), u2 = uniform();
        return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
    }
};

}  // namespace

#define SUR_CU(expr, what)                                                                       \
    do {                                                                                         \
        const cudaError_t e_ = (expr);                                                           \
        if (e_ != cudaSuccess) return set_error(PFB_E_CUDA, "%s: %s", what, cudaGetErrorString(e_)); \
    } while (0)

struct pfb_sur2d {
    int device = 0;
    int max_batch = 0;
    cudaStream_t stream = nullptr;
    long long nparams = 0;
    size_t w_off[8] = {}, b_off[8] = {};
    float* params = nullptr;
    float* grads = nullptr;
    float* adam_m = nullptr;
    float* adam_v = nullptr;
    long long adam_t = 0;
    bf16* wf[8] = {};  // packed forward weights
    bf16* wd[8] = {};  // packed data-gradient weights
    // activations and gradients (padded channels-last), max_batch images
    bf16 *x0 = nullptr, *a1 = nullptr, *a2 = nullptr, *p = nullptr, *a3 = nullptr, *a4 = nullptr,
         *u = nullptr, *a5 = nullptr, *a6 = nullptr, *a7 = nullptr;
    float* out = nullptr;
    bf16 *go = nullptr, *dz7 = nullptr, *dz6 = nullptr, *dz5 = nullptr, *gu = nullptr,
         *dz4 = nullptr, *dz3 = nullptr, *gp = nullptr, *dz2 = nullptr, *dz1 = nullptr;
    float* target = nullptr;
    float* dphi = nullptr;
    int* origins = nullptr;
    double* loss_partial = nullptr;
    float* wg_ws = nullptr;
    size_t wg_bytes = 0;
    std::vector<void*> owned;

    ~pfb_sur2d() {
        for (void* q : owned) cudaFree(q);
        if (stream) cudaStreamDestroy(stream);
    }

    template <typename T>
    int alloc(T** ptr, size_t count) {
        void* q = nullptr;
        SUR_CU(cudaMalloc(&q, count * sizeof(T)), "surrogate alloc");
        owned.push_back(q);
        SUR_CU(cudaMemset(q, 0, count * sizeof(T)), "surrogate memset");
        *ptr = static_cast<T*>(q);
        return PFB_OK;
    }

    int setup(int mb, unsigned long long seed, int dev) {
        device = dev;
        max_batch = mb;
        SUR_CU(cudaSetDevice(dev), "cudaSetDevice");
        SUR_CU(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "stream");
        long long off = 0;
        for (int l = 0; l < 8; ++l) {
            w_off[l] = (size_t)off;
            off += 9LL * kLayers[l].cin * kLayers[l].cout;
            b_off[l] = (size_t)off;
            off += kLayers[l].cout;
        }
        nparams = off;
        int rc;
        if ((rc = alloc(&params, (size_t)nparams)) || (rc = alloc(&grads, (size_t)nparams)) ||
            (rc = alloc(&adam_m, (size_t)nparams)) || (rc = alloc(&adam_v, (size_t)nparams)))
            return rc;
        for (int l = 0; l < 8; ++l) {
            const size_t n = 9 * (size_t)kLayers[l].cin * kLayers[l].cout;
            if ((rc = alloc(&wf[l], n)) || (rc = alloc(&wd[l], n))) return rc;
        }
        const size_t B = (size_t)mb;
        if ((rc = alloc(&x0, B * kP64 * 16)) || (rc = alloc(&a1, B * kP64 * 32)) ||
            (rc = alloc(&a2, B * kP64 * 32)) || (rc = alloc(&p, B * kP32 * 32)) ||
            (rc = alloc(&a3, B * kP32 * 32)) || (rc = alloc(&a4, B * kP32 * 32)) ||
            (rc = alloc(&u, B * kP64 * 32)) || (rc = alloc(&a5, B * kP64 * 32)) ||
            (rc = alloc(&a6, B * kP64 * 32)) || (rc = alloc(&a7, B * kP64 * 32)) ||
            (rc = alloc(&out, B * kP64 * 16)) || (rc = alloc(&go, B * kP64 * 16)) ||
            (rc = alloc(&dz7, B * kP64 * 32)) || (rc = alloc(&dz6, B * kP64 * 32)) ||
            (rc = alloc(&dz5, B * kP64 * 32)) || (rc = alloc(&gu, B * kP64 * 32)) ||
            (rc = alloc(&dz4, B * kP32 * 32)) || (rc = alloc(&dz3, B * kP32 * 32)) ||
            (rc = alloc(&gp, B * kP32 * 32)) || (rc = alloc(&dz2, B * kP64 * 32)) ||
            (rc = alloc(&dz1, B * kP64 * 32)) || (rc = alloc(&target, B * kImg * kImg)) ||
            (rc = alloc(&dphi, B * kImg * kImg)) || (rc = alloc(&origins, B * 2)) ||
            (rc = alloc(&loss_partial, (size_t)kLossBlocks)))
            return rc;
        wg_bytes = conv3x3_wgrad_workspace(mb, kImg, kImg, 32, 32);
        if ((rc = alloc(&wg_ws, wg_bytes / sizeof(float)))) return rc;
        // He-normal weights on the real input channels; the last layer starts
        // at zero (identity jump), padded channels stay zero
        std::vector<float> h((size_t)nparams, 0.0f);
        Rng rng{seed};
        for (int l = 0; l < 7; ++l) {
            const LayerSpec& L = kLayers[l];
            const double sd = std::sqrt(2.0 / (9.0 * L.cin_real));
            for (int co = 0; co < L.cout_real; ++co)
                for (int ci = 0; ci < L.cin_real; ++ci)
                    for (int k = 0; k < 9; ++k)
                        h[w_off[l] + ((size_t)co * L.cin + ci) * 9 + k] = (float)(sd * rng.normal());
        }
        SUR_CU(cudaMemcpy(params, h.data(), h.size() * sizeof(float), cudaMemcpyHostToDevice),
               "upload weights");
        return repack(stream);
    }

    int repack(cudaStream_t s) {
        for (int l = 0; l < 8; ++l) {
            int rc = conv3x3_pack(params + w_off[l], wf[l], kLayers[l].cin, kLayers[l].cout, 0, s);
            if (!rc && l > 0) rc = conv3x3_pack(params + w_off[l], wd[l], kLayers[l].cin, kLayers[l].cout, 1, s);
            if (rc) return rc;
        }
        return PFB_OK;
    }

    int conv(int l, const bf16* in, bf16* o, float* of, int B, cudaStream_t s) {
        const LayerSpec& L = kLayers[l];
        return conv3x3_fwd(in, o, of, wf[l], params + b_off[l], nullptr, B, L.res, L.res, L.cin,
                           L.cout, L.relu, s);
    }
    // data gradient of layer l: dY (cout channels) -> dX (cin), gated by the
    // ReLU of the layer's input when it is one
    int dgrad(int l, const bf16* dy, bf16* dx, const bf16* gate, int B, cudaStream_t s) {
        const LayerSpec& L = kLayers[l];
        return conv3x3_fwd(dy, dx, nullptr, wd[l], nullptr, gate, B, L.res, L.res, L.cout, L.cin, 0, s);
    }
    int wgrad(int l, const bf16* x, const bf16* dy, int B, cudaStream_t s) {
        const LayerSpec& L = kLayers[l];
        return conv3x3_wgrad(x, dy, wg_ws, wg_bytes, grads + w_off[l], grads + b_off[l], B, L.res,
                             L.res, L.cin, L.cout, s);
    }

    int forward(const bf16* in, int B, cudaStream_t s) {
        int rc;
        if ((rc = conv(0, in, a1, nullptr, B, s)) || (rc = conv(1, a1, a2, nullptr, B, s))) return rc;
        k_pool2<<<ew_blocks((long long)B * kHalf * kHalf * 4), kEwThreads, 0, s>>>(
            reinterpret_cast<const uint4*>(a2), reinterpret_cast<uint4*>(p), B);
        if ((rc = conv(2, p, a3, nullptr, B, s)) || (rc = conv(3, a3, a4, nullptr, B, s))) return rc;
        k_upadd<<<ew_blocks((long long)B * kImg * kImg * 4), kEwThreads, 0, s>>>(
            reinterpret_cast<const uint4*>(a4), reinterpret_cast<const uint4*>(a2),
            reinterpret_cast<uint4*>(u), B);
        if ((rc = conv(4, u, a5, nullptr, B, s)) || (rc = conv(5, a5, a6, nullptr, B, s)) ||
            (rc = conv(6, a6, a7, nullptr, B, s)) || (rc = conv(7, a7, nullptr, out, B, s)))
            return rc;
        const cudaError_t e = cudaGetLastError();
        return e == cudaSuccess ? PFB_OK : set_error(PFB_E_CUDA, "forward: %s", cudaGetErrorString(e));
    }

    int backward(int B, cudaStream_t s) {
        int rc;
        if ((rc = wgrad(7, a7, go, B, s)) || (rc = dgrad(7, go, dz7, a7, B, s)) ||
            (rc = wgrad(6, a6, dz7, B, s)) || (rc = dgrad(6, dz7, dz6, a6, B, s)) ||
            (rc = wgrad(5, a5, dz6, B, s)) || (rc = dgrad(5, dz6, dz5, a5, B, s)) ||
            (rc = wgrad(4, u, dz5, B, s)) || (rc = dgrad(4, dz5, gu, nullptr, B, s)))
            return rc;
        k_upback_gate<<<ew_blocks((long long)B * kHalf * kHalf * 4), kEwThreads, 0, s>>>(
            reinterpret_cast<const uint4*>(gu), reinterpret_cast<const uint4*>(a4),
            reinterpret_cast<uint4*>(dz4), B);
        if ((rc = wgrad(3, a3, dz4, B, s)) || (rc = dgrad(3, dz4, dz3, a3, B, s)) ||
            (rc = wgrad(2, p, dz3, B, s)) || (rc = dgrad(2, dz3, gp, nullptr, B, s)))
            return rc;
        k_skipgrad<<<ew_blocks((long long)B * kImg * kImg * 4), kEwThreads, 0, s>>>(
            reinterpret_cast<const uint4*>(gp), reinterpret_cast<const uint4*>(gu),
            reinterpret_cast<const uint4*>(a2), reinterpret_cast<uint4*>(dz2), B);
        if ((rc = wgrad(1, a1, dz2, B, s)) || (rc = dgrad(1, dz2, dz1, a1, B, s)) ||
            (rc = wgrad(0, x0, dz1, B, s)))
            return rc;
        const cudaError_t e = cudaGetLastError();
        return e == cudaSuccess ? PFB_OK : set_error(PFB_E_CUDA, "backward: %s", cudaGetErrorString(e));
    }
};

extern "C" {

pfb_sur2d* pfb_sur2d_create(int max_batch, unsigned long long seed, int device) {
    clear_error();
    if (max_batch < 1 || max_batch > 4096) {
        set_error(PFB_E_ARG, "max_batch must be in 1..4096");
        return nullptr;
    }
    pfb_sur2d* n = new (std::nothrow) pfb_sur2d();
    if (!n) {
        set_error(PFB_E_NOMEM, "host allocation failed");
        return nullptr;
    }
    if (n->setup(max_batch, seed, device) != PFB_OK || cudaStreamSynchronize(n->stream) != cudaSuccess) {
        delete n;
        return nullptr;
    }
    return n;
}

void pfb_sur2d_destroy(pfb_sur2d* n) { delete n; }

long long pfb_sur2d_num_params(const pfb_sur2d* n) { return n ? n->nparams : -1; }

int pfb_sur2d_get_params(pfb_sur2d* n, float* out) {
    if (!n || !out) return set_error(PFB_E_ARG, "get_params: null argument");
    SUR_CU(cudaSetDevice(n->device), "cudaSetDevice");
    SUR_CU(cudaMemcpyAsync(out, n->params, (size_t)n->nparams * sizeof(float),
                           cudaMemcpyDeviceToHost, n->stream), "download params");
    SUR_CU(cudaStreamSynchronize(n->stream), "sync");
    return PFB_OK;
}

int pfb_sur2d_set_params(pfb_sur2d* n, const float* in) {
    if (!n || !in) return set_error(PFB_E_ARG, "set_params: null argument");
    SUR_CU(cudaSetDevice(n->device), "cudaSetDevice");
    SUR_CU(cudaMemcpyAsync(n->params, in, (size_t)n->nparams * sizeof(float),
                           cudaMemcpyHostToDevice, n->stream), "upload params");
    SUR_CU(cudaMemsetAsync(n->adam_m, 0, (size_t)n->nparams * sizeof(float), n->stream), "reset");
    SUR_CU(cudaMemsetAsync(n->adam_v, 0, (size_t)n->nparams * sizeof(float), n->stream), "reset");
    n->adam_t = 0;
    const int rc = n->repack(n->stream);
    if (rc) return rc;
    SUR_CU(cudaStreamSynchronize(n->stream), "sync");
    return PFB_OK;
}

int pfb_sur2d_get_grads(pfb_sur2d* n, float* out) {
    if (!n || !out) return set_error(PFB_E_ARG, "get_grads: null argument");
    SUR_CU(cudaSetDevice(n->device), "cudaSetDevice");
    SUR_CU(cudaMemcpyAsync(out, n->grads, (size_t)n->nparams * sizeof(float),
                           cudaMemcpyDeviceToHost, n->stream), "download grads");
    SUR_CU(cudaStreamSynchronize(n->stream), "sync");
    return PFB_OK;
}

int pfb_sur2d_predict(pfb_sur2d* n, const void* x0, float* dphi, int batch) {
    clear_error();
    if (!n || !x0 || !dphi || batch < 1) return set_error(PFB_E_ARG, "predict: bad argument");
    SUR_CU(cudaSetDevice(n->device), "cudaSetDevice");
    for (int b0 = 0; b0 < batch; b0 += n->max_batch) {
        const int B = batch - b0 < n->max_batch ? batch - b0 : n->max_batch;
        const bf16* in = static_cast<const bf16*>(x0) + (size_t)b0 * kP64 * 16;
        int rc = n->forward(in, B, n->stream);
        if (rc) return rc;
        k_take_ch0<<<ew_blocks((long long)B * kImg * kImg), kEwThreads, 0, n->stream>>>(
            n->out, dphi + (size_t)b0 * kImg * kImg, B);
    }
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? PFB_OK : set_error(PFB_E_CUDA, "predict: %s", cudaGetErrorString(e));
}

// Loss and gradients of one batch without an update (the gradient check).
static int loss_and_grads(pfb_sur2d* n, int B, double* loss) {
    int rc = n->forward(n->x0, B, n->stream);
    if (rc) return rc;
    k_loss<<<kLossBlocks, kEwThreads, 0, n->stream>>>(n->out, n->target, reinterpret_cast<uint4*>(n->go),
                                                      n->loss_partial, B,
                                                      1.0f / (float)((double)B * kImg * kImg));
    rc = n->backward(B, n->stream);
    if (rc) return rc;
    if (loss) {
        double h[kLossBlocks];
        SUR_CU(cudaMemcpyAsync(h, n->loss_partial, sizeof(h), cudaMemcpyDeviceToHost, n->stream),
               "download loss");
        SUR_CU(cudaStreamSynchronize(n->stream), "sync");
        double t = 0.0;
        for (int k = 0; k < kLossBlocks; ++k) t += h[k];
        *loss = t / ((double)B * kImg * kImg);
    }
    return PFB_OK;
}

int pfb_sur2d_loss_grad(pfb_sur2d* n, const void* x_all, const float* t_all, const int* idx,
                        int batch, double* loss) {
    clear_error();
    if (!n || !x_all || !t_all || !idx || batch < 1 || batch > n->max_batch)
        return set_error(PFB_E_ARG, "loss_grad: bad argument");
    SUR_CU(cudaSetDevice(n->device), "cudaSetDevice");
    k_gather<<<batch, kEwThreads, 0, n->stream>>>(static_cast<const uint4*>(x_all), t_all, idx,
                                                  reinterpret_cast<uint4*>(n->x0), n->target);
    return loss_and_grads(n, batch, loss);
}

int pfb_sur2d_train_step(pfb_sur2d* n, const void* x_all, const float* t_all, const int* idx,
                         int batch, float lr, double* loss) {
    int rc = pfb_sur2d_loss_grad(n, x_all, t_all, idx, batch, loss);
    if (rc) return rc;
    n->adam_t += 1;
    const float b1 = 0.9f, b2 = 0.999f;
    const float bc1 = 1.0f - (float)std::pow((double)b1, (double)n->adam_t);
    const float bc2 = 1.0f - (float)std::pow((double)b2, (double)n->adam_t);
    k_adam<<<ew_blocks(n->nparams), kEwThreads, 0, n->stream>>>(n->params, n->grads, n->adam_m,
                                                                n->adam_v, n->nparams, lr, b1, b2,
                                                                1e-8f, bc1, bc2);
    rc = n->repack(n->stream);
    if (rc) return rc;
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? PFB_OK : set_error(PFB_E_CUDA, "train_step: %s", cudaGetErrorString(e));
}

int pfb_sur2d_sync(pfb_sur2d* n) {
    if (!n) return set_error(PFB_E_ARG, "null surrogate");
    SUR_CU(cudaStreamSynchronize(n->stream), "sync");
    return PFB_OK;
}

// Jump every cell of `s` by the network: crops of the current state (with
// the rate over the last history_steps plain steps, taken here, when
// history_steps > 0), the predicted increments added back into the cells'
// tiles, then moments and aggregate rebuilt. Runs on the system's stream.
int pfb_sur2d_jump_history(pfb_sur2d* n, pfb_sim2d* s, int history_steps, float hist_scale) {
    clear_error();
    if (!n || !s || history_steps < 0) return set_error(PFB_E_ARG, "jump: bad argument");
    Sim2DView v;
    int rc = sim2d_view(s, &v);
    if (rc) return rc;
    if (v.device != n->device) return set_error(PFB_E_CONFIG, "jump: system and network on different devices");
    SUR_CU(cudaSetDevice(n->device), "cudaSetDevice");
    const int N = v.N;
    bf16* xin = nullptr;
    float* d = nullptr;
    int* org = nullptr;
    SUR_CU(cudaMallocAsync(&xin, (size_t)N * kP64 * 16 * sizeof(bf16), v.stream), "jump alloc");
    SUR_CU(cudaMallocAsync(&d, (size_t)N * kImg * kImg * sizeof(float), v.stream), "jump alloc");
    SUR_CU(cudaMallocAsync(&org, (size_t)N * 2 * sizeof(int), v.stream), "jump alloc");
    float* prev = nullptr;
    if (history_steps > 0) {
        SUR_CU(cudaMallocAsync(&prev, (size_t)N * kImg * kImg * sizeof(float), v.stream), "jump alloc");
        rc = relax_extract(s, xin, prev, org, nullptr, nullptr, 0.0f);
        if (!rc) rc = pfb_sim2d_advance(s, history_steps);
        if (!rc) rc = relax_extract(s, xin, nullptr, nullptr, org, prev, hist_scale);
    } else {
        rc = relax_extract(s, xin, nullptr, org, nullptr, nullptr, 0.0f);
    }
    for (int b0 = 0; !rc && b0 < N; b0 += n->max_batch) {
        const int B = N - b0 < n->max_batch ? N - b0 : n->max_batch;
        rc = n->forward(xin + (size_t)b0 * kP64 * 16, B, v.stream);
        if (!rc)
            k_take_ch0<<<ew_blocks((long long)B * kImg * kImg), kEwThreads, 0, v.stream>>>(
                n->out, d + (size_t)b0 * kImg * kImg, B);
    }
    if (!rc) rc = relax_insert(s, org, d);
    cudaFreeAsync(xin, v.stream);
    cudaFreeAsync(d, v.stream);
    cudaFreeAsync(org, v.stream);
    if (prev) cudaFreeAsync(prev, v.stream);
    const cudaError_t e = cudaStreamSynchronize(v.stream);
    if (rc) return rc;
    SUR_CU(e, "jump sync");
    return PFB_OK;
}

int pfb_sur2d_jump(pfb_sur2d* n, pfb_sim2d* s) { return pfb_sur2d_jump_history(n, s, 0, 0.0f); }

// Device time of `iters` forward passes over `batch` images (inputs as they
// are in the network's buffer), ms per pass.
int pfb_sur2d_bench_forward(pfb_sur2d* n, int batch, int iters, double* ms) {
    clear_error();
    if (!n || batch < 1 || batch > n->max_batch || iters < 1 || !ms)
        return set_error(PFB_E_ARG, "bench_forward: bad argument");
    SUR_CU(cudaSetDevice(n->device), "cudaSetDevice");
    int rc = n->forward(n->x0, batch, n->stream);
    if (rc) return rc;
    cudaEvent_t e0, e1;
    SUR_CU(cudaEventCreate(&e0), "event");
    SUR_CU(cudaEventCreate(&e1), "event");
    cudaEventRecord(e0, n->stream);
    for (int i = 0; i < iters && !rc; ++i) rc = n->forward(n->x0, batch, n->stream);
    cudaEventRecord(e1, n->stream);
    const cudaError_t e = cudaEventSynchronize(e1);
    float t = 0.0f;
    cudaEventElapsedTime(&t, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    SUR_CU(e, "bench sync");
    *ms = (double)t / iters;
    return PFB_OK;
}

}  // extern "C"
