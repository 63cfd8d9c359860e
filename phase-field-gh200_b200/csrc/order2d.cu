// Morton visit order of the 2D cells (the reference's --morton: src/sim.cu:
// 284-296 and 649-653, src/kernels.cu:1267-1305). Every sixth step the cells
// are ordered by the Z-order index of their centroid pixel, so that clusters
// launched together update neighbouring windows and share S rows in L2. The
// order changes no result: a cell's update reads the previous step's S and
// its own phi, and scatters into S with integer atomics.
//
// Key of cell i: (morton(cx, cy) << 32) | i, where (cx, cy) is the window
// origin plus the truncated centroid offset (Cx / V, Cy / V; V <= 0 counts as
// 1), wrapped into [0, L). Keys are distinct, so the order is unique and the
// same as the reference's. One CTA sorts the keys in shared memory with
// Batcher's bitonic network over the next power of two M >= N (padding keys
// are all ones and sort last).
#include <cuda_runtime.h>

#include <mutex>

#include <cstdint>

#include "pfb200.h"
#include "pfb_common.cuh"

namespace pfb {
namespace {

constexpr int kOrderThreads = 1024;

__device__ __forceinline__ uint32_t spread_bits(uint32_t v) {
    v &= 0x0000FFFFu;
    v = (v | (v << 8)) & 0x00FF00FFu;
    v = (v | (v << 4)) & 0x0F0F0F0Fu;
    v = (v | (v << 2)) & 0x33333333u;
    v = (v | (v << 1)) & 0x55555555u;
    return v;
}

__device__ __forceinline__ int wrap_side(int v, int L) {
    v %= L;
    return v < 0 ? v + L : v;
}

__global__ void __launch_bounds__(kOrderThreads) k_visit_order2d(const pfb_cell2d* __restrict__ cell,
                                                                  uint32_t* __restrict__ perm, int N, int M,
                                                                  int L) {
    extern __shared__ unsigned long long keys[];
    for (int i = threadIdx.x; i < M; i += blockDim.x) {
        unsigned long long k = ~0ull;
        if (i < N) {
            const pfb_cell2d c = cell[i];
            const double V = c.V > 0.0 ? c.V : 1.0;
            const uint32_t cx = (uint32_t)wrap_side(c.gx0 + (int)(c.Cx / V), L);
            const uint32_t cy = (uint32_t)wrap_side(c.gy0 + (int)(c.Cy / V), L);
            k = ((unsigned long long)(spread_bits(cx) | (spread_bits(cy) << 1)) << 32) | (uint32_t)i;
        }
        keys[i] = k;
    }
    __syncthreads();
    // Bitonic merge: blocks of size `span` alternate ascending and descending
    // until the last merge, which is ascending over all M keys.
    for (int span = 2; span <= M; span <<= 1) {
        for (int gap = span >> 1; gap > 0; gap >>= 1) {
            for (int i = threadIdx.x; i < M; i += blockDim.x) {
                const int partner = i ^ gap;
                if (partner <= i) continue;
                const unsigned long long a = keys[i], b = keys[partner];
                const bool ascending = (i & span) == 0;
                if ((a > b) == ascending) {
                    keys[i] = b;
                    keys[partner] = a;
                }
            }
            __syncthreads();
        }
    }
    for (int i = threadIdx.x; i < N; i += blockDim.x) perm[i] = (uint32_t)keys[i];
}

}  // namespace

// Largest cell count one sorting CTA holds (M * 8 bytes of shared memory).
int visit_order2d_capacity() {
    int dev = 0, optin = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess)
        optin = 227 * 1024;
    int m = 1;
    while ((size_t)(m << 1) * sizeof(unsigned long long) <= (size_t)optin) m <<= 1;
    return m;
}

// Shared-memory opt-in for up to N cells; call outside stream capture. The
// attribute belongs to the kernel on the whole device, so it only ever grows
// (a smaller system created later must not shrink it under a larger one).
cudaError_t visit_order2d_prepare(int N) {
    static std::mutex mu;
    static int granted[64] = {};
    int M = 1;
    while (M < N) M <<= 1;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const int bytes = (int)(M * sizeof(unsigned long long));
    std::lock_guard<std::mutex> lock(mu);
    if (dev >= 0 && dev < 64 && granted[dev] >= bytes) return cudaSuccess;
    e = cudaFuncSetAttribute(k_visit_order2d, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess && dev >= 0 && dev < 64) granted[dev] = bytes;
    return e;
}

cudaError_t visit_order2d_launch(const pfb_cell2d* cell, uint32_t* perm, int N, int L, cudaStream_t stream) {
    int M = 1;
    while (M < N) M <<= 1;
    k_visit_order2d<<<1, kOrderThreads, (size_t)M * sizeof(unsigned long long), stream>>>(cell, perm, N, M, L);
    return cudaGetLastError();
}

}  // namespace pfb
