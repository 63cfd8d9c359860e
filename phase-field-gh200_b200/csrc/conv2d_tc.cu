// 3x3 "same" convolutions on bfloat16 activations with binary32
// accumulation on the tcgen05 tensor cores: forward (and data gradient, the
// same kernel with flipped, transposed weights) and weight gradient. These
// are the contractions of the learned relaxation surrogate; nothing here has
// a counterpart in the reference.
//
// Activation layout ("padded NHWC"): image b of H x W pixels with C channels
// is stored as (H + 2) x (W + 2) positions q = yp (W + 2) + xp, channels
// innermost, with a one-pixel zero border (yp = 0, H + 1 or xp = 0, W + 1).
// A tap (dy, dx) of the 3x3 stencil is then a constant offset
// off = dy (W + 2) + dx in q, and a run of 128 consecutive q is one GEMM
// M-tile whose rows keep a uniform stride even across image rows: outputs at
// the border columns are computed and discarded (2 of W + 2 columns).
//
// Forward: out[q][co] = sum_tap sum_ci in[q + off_tap][ci] W[co][ci][tap],
// an implicit GEMM with M = 128 positions, N = Cout, K = 9 Cin. The input
// rows of a CTA's M-tiles plus the stencil halo are staged once in shared
// memory as Cin/8 "chunk planes" (plane c holds channels 8c..8c+7 of every
// staged position, 16 B per position), which is the K-major core-matrix
// layout for every tap at once: tap (dy, dx) only moves the descriptor's
// start row. Weights are pre-packed in global memory in the same layout.
//
// Weight gradient: dW[co][ci][tap] = sum_q dY[q][co] in[q + off_tap][ci],
// K = positions. Both operands are MN-major chunk planes (8 channels of one
// position per 16 B); the M dimension (128 rows) packs 128 / Cin taps, each
// tap's planes holding the input shifted by that tap's offset. A slot of
// ones after the nine taps yields the bias gradient sum_q dY[q][co] from the
// same MMAs. Each CTA reduces a range of positions of one image into TMEM
// and writes its partial sums; a second kernel adds the partials in a fixed
// order, so the result is deterministic.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <cstdint>
#include <mutex>

#include "pfb_internal.h"
#include "tc_util.cuh"
#include "pfb200_surrogate.h"

namespace pfb {
namespace {

__device__ unsigned int g_conv_status = 0u;  // bit 0: an MMA completion wait gave up

using bf16 = __nv_bfloat16;

constexpr int kConvThreads = 128;  // 4 warps: one TMEM lane quadrant each
constexpr int kConvMT = 2;         // M-tiles (of 128 positions) per forward CTA
constexpr int kWgKT = 64;          // positions per weight-gradient K chunk

__host__ __device__ constexpr int round_up(int v, int m) { return (v + m - 1) / m * m; }

// Rows staged for a forward CTA: its MT x 128 positions plus the halo.
__host__ __device__ constexpr int fwd_rows(int W) { return kConvMT * 128 + 2 * (W + 2) + 2; }
// Chunk-plane stride in bytes; 32 mod 128 spreads the staging stores of the
// four planes of one position over distinct banks.
__host__ __device__ constexpr int fwd_plane(int W) { return round_up(fwd_rows(W) * 16, 128) + 32; }

template <int CIN, int COUT>
__host__ __device__ constexpr int fwd_smem(int W) {
    return (CIN / 8) * fwd_plane(W) + 9 * (CIN / 8) * COUT * 16 + 16;
}

template <int COUT>
__host__ __device__ constexpr uint32_t fwd_tmem_cols() {
    return kConvMT * COUT <= 32 ? 32u : kConvMT * COUT <= 64 ? 64u : 128u;
}

struct ConvFwdArgs {
    const bf16* x;     // [B][P2][CIN]
    bf16* y;           // [B][P2][COUT] or null
    float* yf;         // [B][P2][COUT] or null (binary32 copy of the output)
    const bf16* w;     // packed [9][CIN / 8][COUT][8]
    const float* bias; // [COUT] or null
    const bf16* gate;  // [B][P2][COUT] or null: output *= (gate > 0)
    int B, H, W;
    int relu;
    int tiles;  // CTAs per image
};

template <int CIN, int COUT>
__global__ void __launch_bounds__(kConvThreads) k_conv3x3_fwd(const __grid_constant__ ConvFwdArgs A) {
    static_assert(CIN % 16 == 0 && COUT % 16 == 0 && COUT <= 64, "channel counts");
    constexpr int NCA = CIN / 8;
    constexpr uint32_t NCOLS = fwd_tmem_cols<COUT>();
    extern __shared__ __align__(128) unsigned char smem[];
    const int W2 = A.W + 2;
    const int P2 = (A.H + 2) * W2;
    const int CH = fwd_plane(A.W);
    const int RA = fwd_rows(A.W);
    unsigned char* sA = smem;
    unsigned char* sW = smem + NCA * CH;
    uint64_t* bar = reinterpret_cast<uint64_t*>(sW + 9 * NCA * COUT * 16);
    uint32_t* slot = reinterpret_cast<uint32_t*>(bar + 1);

    const int tid = (int)threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    const int b = (int)blockIdx.x / A.tiles;
    const int tile = (int)blockIdx.x - b * A.tiles;
    const int q0 = W2 + tile * (kConvMT * 128);  // first output position
    const int qa = q0 - (W2 + 1);                // first staged position
    const int q_end = (A.H + 1) * W2;            // one past the last interior row

    if (tid == 0) dev::mbar_init(bar, 1);
    if (warp == 0) {
        tc::tmem_alloc(slot, NCOLS);
        tc::tmem_relinquish();
    }
    // stage the input rows (zero outside the image) and the packed weights
    const bf16* xb = A.x + (size_t)b * P2 * CIN;
    const uint32_t sa = dev::smem_addr(sA);
    for (int u = tid; u < RA * NCA; u += kConvThreads) {
        const int row = u / NCA, c = u - row * NCA;
        const int q = qa + row;
        const bool ok = q >= 0 && q < P2;
        tc::cp_async16(sa + (uint32_t)(c * CH + row * 16), xb + (size_t)(ok ? q : 0) * CIN + c * 8,
                       ok ? 16u : 0u);
    }
    const uint32_t sw = dev::smem_addr(sW);
    for (int u = tid; u < 9 * NCA * COUT; u += kConvThreads)
        tc::cp_async16(sw + (uint32_t)u * 16u, A.w + (size_t)u * 8, 16u);
    tc::cp_async_wait_all();
    tc::fence_proxy_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *slot;

    if (tid == 0) {
        constexpr uint32_t idesc = tc::idesc_bf16_f32(128, COUT, false, false);
        for (int m = 0; m < kConvMT; ++m) {
            for (int tap = 0; tap < 9; ++tap) {
                const int dy = tap / 3, dx = tap - 3 * (tap / 3);
                const int row = m * 128 + dy * W2 + dx;
                for (int ks = 0; ks < CIN / 16; ++ks) {
                    const uint64_t ad = tc::smem_desc(sa + (uint32_t)(2 * ks * CH + row * 16),
                                                      (uint32_t)CH, 128u);
                    const uint64_t bd = tc::smem_desc(
                        sw + (uint32_t)((tap * NCA + 2 * ks) * COUT * 16), (uint32_t)(COUT * 16), 128u);
                    tc::mma_bf16(tmem + (uint32_t)(m * COUT), ad, bd, idesc, (tap | ks) ? 1u : 0u);
                }
            }
        }
        tc::mma_commit(bar);
    }
    // every thread takes the same branch (the TMEM loads are warp-collective)
    const bool done = __syncthreads_and(dev::mbar_wait_bounded(bar, 0, tc::kMmaWaitPolls)) != 0;
    tc::fence_after_sync();
    if (!done) {
        if (tid == 0) atomicOr(&g_conv_status, 1u);
    } else {
        const int r = warp * 32 + lane;
        for (int m = 0; m < kConvMT; ++m) {
            float acc[COUT];
            __syncwarp();
#pragma unroll
            for (int h = 0; h < COUT / 16; ++h) {
                uint32_t v[16];
                tc::tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(m * COUT + 16 * h), v);
                tc::tmem_wait_ld();
#pragma unroll
                for (int j = 0; j < 16; ++j) acc[16 * h + j] = __uint_as_float(v[j]);
            }
            const int q = q0 + m * 128 + r;
            if (q < q_end) {
            const int xp = q % W2;
            const bool interior = xp >= 1 && xp <= A.W;
            const size_t o = ((size_t)b * P2 + q) * COUT;
            float g[COUT];
#pragma unroll
            for (int j = 0; j < COUT; ++j) g[j] = 1.0f;
            if (A.gate && interior) {
#pragma unroll
                for (int h = 0; h < COUT / 8; ++h) {
                    const uint4 gv = *reinterpret_cast<const uint4*>(A.gate + o + 8 * h);
                    const bf16* ge = reinterpret_cast<const bf16*>(&gv);
#pragma unroll
                    for (int j = 0; j < 8; ++j) g[8 * h + j] = __bfloat162float(ge[j]) > 0.0f ? 1.0f : 0.0f;
                }
            }
#pragma unroll
            for (int j = 0; j < COUT; ++j) {
                float v = acc[j];
                if (A.bias) v += A.bias[j];
                if (A.relu) v = fmaxf(v, 0.0f);
                v *= g[j];
                acc[j] = interior ? v : 0.0f;
            }
            if (A.y) {
#pragma unroll
                for (int h = 0; h < COUT / 8; ++h) {
                    uint4 pk;
                    __nv_bfloat162* p2 = reinterpret_cast<__nv_bfloat162*>(&pk);
#pragma unroll
                    for (int j = 0; j < 4; ++j)
                        p2[j] = __floats2bfloat162_rn(acc[8 * h + 2 * j], acc[8 * h + 2 * j + 1]);
                    *reinterpret_cast<uint4*>(A.y + o + 8 * h) = pk;
                }
            }
            if (A.yf) {
#pragma unroll
                for (int h = 0; h < COUT / 4; ++h)
                    *reinterpret_cast<float4*>(A.yf + o + 4 * h) =
                        make_float4(acc[4 * h], acc[4 * h + 1], acc[4 * h + 2], acc[4 * h + 3]);
            }
            }
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, NCOLS);
}

// ---- forward, persistent and warp-specialised ----------------------------------
// The same contraction as k_conv3x3_fwd with the three stages of a tile in
// separate warps so that they overlap across tiles: warp 0 loads a tile's
// chunk planes with TMA (cp.async.bulk.tensor, a 4D view of the activations:
// 8 channels x channel chunk x position x image, so positions outside the
// image arrive as zeros) into a two-stage ring; warp 1 issues the tile's
// tcgen05 MMAs into one of two TMEM accumulators and commits; warps 2-5
// (one TMEM lane quadrant each) run the epilogue of the previous tile. The
// packed weights are staged once per CTA with one bulk copy. Each CTA walks
// tiles c, c + G, c + 2G, ... of the B x tiles work list.
constexpr int kWsThreads = 192;
constexpr int kWsStages = 2;

// rows per TMA box: half the staged rows, rounded up to 8 (two boxes per plane)
__host__ __device__ constexpr int ws_box(int W) { return round_up((fwd_rows(W) + 1) / 2, 8); }
__host__ __device__ constexpr int ws_plane(int W) { return round_up(2 * ws_box(W) * 16, 128); }

template <int CIN, int COUT>
__host__ __device__ constexpr int ws_smem(int W) {
    return 1024 + kWsStages * (CIN / 8) * ws_plane(W) + 9 * (CIN / 8) * COUT * 16;
}

struct WsHeader {
    uint64_t full[kWsStages], empty[kWsStages], acc_full[2], acc_empty[2], wbar;
    uint32_t tmem_slot;
    int fail;
};

__device__ __forceinline__ void tma_load4(uint32_t dst, const CUtensorMap* map, int c0, int c1, int c2,
                                          int c3, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes "
        "[%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(bar)
        : "memory");
}

template <int CIN, int COUT>
__global__ void __launch_bounds__(kWsThreads)
    k_conv3x3_fwd_ws(const __grid_constant__ ConvFwdArgs A, const __grid_constant__ CUtensorMap X) {
    static_assert(CIN % 16 == 0 && COUT % 16 == 0 && COUT <= 64, "channel counts");
    constexpr int NCA = CIN / 8;
    constexpr uint32_t NCOLS = 2 * fwd_tmem_cols<COUT>();  // two accumulators
    constexpr uint32_t ACC = fwd_tmem_cols<COUT>();
    extern __shared__ __align__(1024) unsigned char smem[];
    WsHeader& H = *reinterpret_cast<WsHeader*>(smem);
    const int W2 = A.W + 2;
    const int P2 = (A.H + 2) * W2;
    const int CH = ws_plane(A.W);
    const int BOX = ws_box(A.W);
    unsigned char* sA = smem + 1024;                                // stages x planes
    unsigned char* sW = sA + (size_t)kWsStages * NCA * CH;          // packed weights
    const uint32_t sa = dev::smem_addr(sA), sw = dev::smem_addr(sW);
    const uint32_t stage_bytes = (uint32_t)(NCA * 2 * BOX * 16);
    const uint32_t wbytes = (uint32_t)(9 * NCA * COUT * 16);

    const int tid = (int)threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int items = A.B * A.tiles;
    const int q_end = (A.H + 1) * W2;

    // every TMA destination below is 128-byte aligned when the dynamic
    // shared memory is; refuse to run otherwise
    if (dev::smem_addr(smem) & 127u) {
        if (tid == 0) atomicOr(&g_conv_status, 2u);
        return;
    }
    if (tid == 0) {
        for (int s = 0; s < kWsStages; ++s) {
            dev::mbar_init(&H.full[s], 1);
            dev::mbar_init(&H.empty[s], 1);
        }
        for (int a = 0; a < 2; ++a) {
            dev::mbar_init(&H.acc_full[a], 1);
            dev::mbar_init(&H.acc_empty[a], 4);  // one arrival per epilogue warp
        }
        dev::mbar_init(&H.wbar, 1);
        H.fail = 0;
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        dev::mbar_arrive_expect_tx(&H.wbar, wbytes);
        dev::bulk_g2s(sW, A.w, wbytes, &H.wbar);
    }
    if (warp == 0) {
        tc::tmem_alloc(&H.tmem_slot, NCOLS);
        tc::tmem_relinquish();
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = H.tmem_slot;
    auto give_up = [&]() {
        H.fail = 1;
        atomicOr(&g_conv_status, 1u);
    };

    if (warp == 0 && lane == 0) {
        // ---- producer: chunk planes of each tile, two boxes per plane
        int k = 0;
        for (int it = (int)blockIdx.x; it < items && !H.fail; it += (int)gridDim.x, ++k) {
            const int s = k % kWsStages;
            if (!dev::mbar_wait_bounded(&H.empty[s], (uint32_t)(((k / kWsStages) & 1) ^ 1), tc::kMmaWaitPolls)) {
                give_up();
                break;
            }
            const int b = it / A.tiles, t = it - b * A.tiles;
            const int qa = t * (kConvMT * 128) - 1;  // first staged position (W2 + t 256 - (W2 + 1))
            const uint32_t bar = dev::smem_addr(&H.full[s]);
            dev::mbar_arrive_expect_tx(&H.full[s], stage_bytes);
            for (int c = 0; c < NCA; ++c)
                for (int h = 0; h < 2; ++h)
                    tma_load4(sa + (uint32_t)((s * NCA + c) * CH + h * BOX * 16), &X, 0, c, qa + h * BOX, b,
                              bar);
        }
        // no copy may still target shared memory at exit
        for (int j = (k > kWsStages ? k - kWsStages : 0); j < k; ++j)
            (void)dev::mbar_wait_bounded(&H.full[j % kWsStages], (uint32_t)((j / kWsStages) & 1),
                                         tc::kMmaWaitPolls);
    } else if (warp == 1 && lane == 0) {
        // ---- MMA issue
        if (!dev::mbar_wait_bounded(&H.wbar, 0, tc::kMmaWaitPolls)) give_up();
        constexpr uint32_t idesc = tc::idesc_bf16_f32(128, COUT, false, false);
        int k = 0;
        for (int it = (int)blockIdx.x; it < items && !H.fail; it += (int)gridDim.x, ++k) {
            const int s = k % kWsStages, a = k & 1;
            if (!dev::mbar_wait_bounded(&H.full[s], (uint32_t)((k / kWsStages) & 1), tc::kMmaWaitPolls) ||
                !dev::mbar_wait_bounded(&H.acc_empty[a], (uint32_t)(((k >> 1) & 1) ^ 1), tc::kMmaWaitPolls)) {
                give_up();
                break;
            }
            tc::fence_after_sync();
            const uint32_t st = sa + (uint32_t)(s * NCA * CH);
            for (int m = 0; m < kConvMT; ++m)
                for (int tap = 0; tap < 9; ++tap) {
                    const int dy = tap / 3, dx = tap - 3 * (tap / 3);
                    const int row = m * 128 + dy * W2 + dx;
                    for (int ks = 0; ks < CIN / 16; ++ks) {
                        const uint64_t ad =
                            tc::smem_desc(st + (uint32_t)(2 * ks * CH + row * 16), (uint32_t)CH, 128u);
                        const uint64_t bd = tc::smem_desc(sw + (uint32_t)((tap * NCA + 2 * ks) * COUT * 16),
                                                          (uint32_t)(COUT * 16), 128u);
                        tc::mma_bf16(tmem + (uint32_t)(a * ACC + m * COUT), ad, bd, idesc,
                                     (tap | ks) ? 1u : 0u);
                    }
                }
            tc::mma_commit(&H.empty[s]);     // the stage may be refilled
            tc::mma_commit(&H.acc_full[a]);  // the accumulator may be read
        }
        // no MMA may still be writing TMEM when it is released
        if (k > 0)
            (void)dev::mbar_wait_bounded(&H.acc_full[(k - 1) & 1], (uint32_t)(((k - 1) >> 1) & 1),
                                         tc::kMmaWaitPolls);
    } else if (warp >= 2) {
        // ---- epilogue: TMEM lane quadrant warp % 4
        const int quad = warp & 3;
        const int r = quad * 32 + lane;
        int k = 0;
        for (int it = (int)blockIdx.x; it < items; it += (int)gridDim.x, ++k) {
            const int a = k & 1;
            const bool ok = dev::mbar_wait_bounded(&H.acc_full[a], (uint32_t)((k >> 1) & 1), tc::kMmaWaitPolls);
            if (!__all_sync(0xFFFFFFFFu, ok) || H.fail) {
                if (lane == 0 && !ok) give_up();
                break;
            }
            tc::fence_after_sync();
            const int b = it / A.tiles, t = it - b * A.tiles;
            const int q0 = W2 + t * (kConvMT * 128);
            for (int m = 0; m < kConvMT; ++m) {
                float acc[COUT];
                __syncwarp();  // the TMEM loads are warp-collective
#pragma unroll
                for (int h = 0; h < COUT / 16; ++h) {
                    uint32_t v[16];
                    tc::tmem_ld16(tmem + ((uint32_t)(quad * 32) << 16) + (uint32_t)(a * ACC + m * COUT + 16 * h), v);
                    tc::tmem_wait_ld();
#pragma unroll
                    for (int j = 0; j < 16; ++j) acc[16 * h + j] = __uint_as_float(v[j]);
                }
                const int q = q0 + m * 128 + r;
                if (q >= q_end) continue;
                const int xp = q % W2;
                const bool interior = xp >= 1 && xp <= A.W;
                const size_t o = ((size_t)b * P2 + q) * COUT;
                float g[COUT];
#pragma unroll
                for (int j = 0; j < COUT; ++j) g[j] = 1.0f;
                if (A.gate && interior) {
#pragma unroll
                    for (int h = 0; h < COUT / 8; ++h) {
                        const uint4 gv = *reinterpret_cast<const uint4*>(A.gate + o + 8 * h);
                        const bf16* ge = reinterpret_cast<const bf16*>(&gv);
#pragma unroll
                        for (int j = 0; j < 8; ++j) g[8 * h + j] = __bfloat162float(ge[j]) > 0.0f ? 1.0f : 0.0f;
                    }
                }
#pragma unroll
                for (int j = 0; j < COUT; ++j) {
                    float v = acc[j];
                    if (A.bias) v += A.bias[j];
                    if (A.relu) v = fmaxf(v, 0.0f);
                    v *= g[j];
                    acc[j] = interior ? v : 0.0f;
                }
                if (A.y) {
#pragma unroll
                    for (int h = 0; h < COUT / 8; ++h) {
                        uint4 pk;
                        __nv_bfloat162* p2 = reinterpret_cast<__nv_bfloat162*>(&pk);
#pragma unroll
                        for (int j = 0; j < 4; ++j)
                            p2[j] = __floats2bfloat162_rn(acc[8 * h + 2 * j], acc[8 * h + 2 * j + 1]);
                        *reinterpret_cast<uint4*>(A.y + o + 8 * h) = pk;
                    }
                }
                if (A.yf) {
#pragma unroll
                    for (int h = 0; h < COUT / 4; ++h)
                        *reinterpret_cast<float4*>(A.yf + o + 4 * h) =
                            make_float4(acc[4 * h], acc[4 * h + 1], acc[4 * h + 2], acc[4 * h + 3]);
                }
            }
            // the accumulator is free again
            tc::fence_before_sync();
            __syncwarp();
            if (lane == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(dev::smem_addr(&H.acc_empty[a])) : "memory");
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, NCOLS);
}

// ---- weight gradient --------------------------------------------------------

template <int CX>
__host__ __device__ constexpr int wg_taps_per_tile() { return 128 / CX; }
template <int CX>
__host__ __device__ constexpr int wg_tiles() { return (10 + 128 / CX - 1) / (128 / CX); }

template <int CX, int CY>
__host__ __device__ constexpr int wg_smem() {
    return wg_tiles<CX>() * 16 * kWgKT * 16 + (CY / 8) * kWgKT * 16 + 16;
}

template <int CY>
__host__ __device__ constexpr uint32_t wg_tmem_cols(int tiles) {
    return tiles * CY <= 32 ? 32u : tiles * CY <= 64 ? 64u : 128u;
}

struct ConvWgradArgs {
    const bf16* x;   // [B][P2][CX] layer input
    const bf16* dy;  // [B][P2][CY] gradient of the layer output (zero border)
    float* partial;  // [grid][9 * CY * CX + CY]
    int B, H, W;
    int ctas;        // CTAs per image
    int chunks;      // K chunks of kWgKT positions per CTA
};

template <int CX, int CY>
__global__ void __launch_bounds__(kConvThreads) k_conv3x3_wgrad(const __grid_constant__ ConvWgradArgs A) {
    static_assert(CX % 16 == 0 && CY % 16 == 0 && CY <= 64, "channel counts");
    constexpr int NCX = CX / 8, NCY = CY / 8;
    constexpr int TPT = wg_taps_per_tile<CX>();
    constexpr int NT = wg_tiles<CX>();
    constexpr uint32_t NCOLS = wg_tmem_cols<CY>(NT);
    constexpr int PLANE = kWgKT * 16;  // bytes per chunk plane
    extern __shared__ __align__(128) unsigned char smem[];
    unsigned char* sA = smem;                     // NT * 16 planes
    unsigned char* sB = smem + NT * 16 * PLANE;   // NCY planes
    uint64_t* bar = reinterpret_cast<uint64_t*>(sB + NCY * PLANE);
    uint32_t* slot = reinterpret_cast<uint32_t*>(bar + 1);

    const int tid = (int)threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    const int W2 = A.W + 2;
    const int P2 = (A.H + 2) * W2;
    const int q_end = (A.H + 1) * W2;
    const int nq = A.H * W2;
    const int b = (int)blockIdx.x / A.ctas;
    const int part = (int)blockIdx.x - b * A.ctas;
    const int total_chunks = (nq + kWgKT - 1) / kWgKT;
    const int c_begin = part * A.chunks;
    const int c_end = min(total_chunks, c_begin + A.chunks);

    if (tid == 0) dev::mbar_init(bar, 1);
    if (warp == 0) {
        tc::tmem_alloc(slot, NCOLS);
        tc::tmem_relinquish();
    }
    // constant slots: slot 9 is all ones (bias gradient), later slots zero
    for (int u = tid; u < (NT * TPT - 9) * NCX * kWgKT; u += kConvThreads) {
        const int plane = 9 * NCX + u / kWgKT, k = u - (u / kWgKT) * kWgKT;
        const uint32_t v = plane < 10 * NCX ? 0x3F803F80u : 0u;
        *reinterpret_cast<uint4*>(sA + plane * PLANE + k * 16) = make_uint4(v, v, v, v);
    }
    const bf16* xb = A.x + (size_t)b * P2 * CX;
    const bf16* yb = A.dy + (size_t)b * P2 * CY;
    const uint32_t sa = dev::smem_addr(sA), sb = dev::smem_addr(sB);
    constexpr uint32_t idesc = tc::idesc_bf16_f32(128, CY, true, true);
    uint32_t tmem = 0;
    bool ok = true;
    int it = 0;
    for (int ck = c_begin; ck < c_end; ++ck, ++it) {
        const int qk = W2 + ck * kWgKT;
        for (int u = tid; u < 9 * NCX * kWgKT; u += kConvThreads) {
            const int k = u % kWgKT, pc = u / kWgKT;  // pc = tap * NCX + c
            const int tap = pc / NCX, c = pc - tap * NCX;
            const int q = qk + k + (tap / 3 - 1) * W2 + (tap % 3 - 1);
            const bool in = q >= 0 && q < P2;
            tc::cp_async16(sa + (uint32_t)(pc * PLANE + k * 16), xb + (size_t)(in ? q : 0) * CX + c * 8,
                           in ? 16u : 0u);
        }
        for (int u = tid; u < NCY * kWgKT; u += kConvThreads) {
            const int k = u % kWgKT, c = u / kWgKT;
            const int q = qk + k;
            const bool in = q < q_end;
            tc::cp_async16(sb + (uint32_t)(c * PLANE + k * 16), yb + (size_t)(in ? q : 0) * CY + c * 8,
                           in ? 16u : 0u);
        }
        tc::cp_async_wait_all();
        tc::fence_proxy_async_smem();
        tc::fence_before_sync();
        __syncthreads();
        tc::fence_after_sync();
        if (it == 0) tmem = *slot;
        if (tid == 0) {
            for (int t = 0; t < NT; ++t)
                for (int kk = 0; kk < kWgKT / 16; ++kk) {
                    const uint64_t ad = tc::smem_desc(sa + (uint32_t)(t * 16 * PLANE + kk * 256), 128u,
                                                      (uint32_t)PLANE);
                    const uint64_t bd = tc::smem_desc(sb + (uint32_t)(kk * 256), 128u, (uint32_t)PLANE);
                    tc::mma_bf16(tmem + (uint32_t)(t * CY), ad, bd, idesc, (it | kk) ? 1u : 0u);
                }
            tc::mma_commit(bar);
        }
        // uniform across the CTA: a partial exit would strand the barriers
        if (!__syncthreads_and(dev::mbar_wait_bounded(bar, (uint32_t)(it & 1), tc::kMmaWaitPolls))) {
            ok = false;
            break;
        }
        tc::fence_after_sync();
    }
    if (it == 0) {  // no chunk for this CTA (not launched that way; kept total)
        tc::fence_before_sync();
        __syncthreads();
        tc::fence_after_sync();
        tmem = *slot;
    }
    float* out = A.partial + (size_t)blockIdx.x * (9 * CY * CX + CY);
    if (!ok) {
        // the MMA wait gave up: poison this CTA's block so the reduction
        // yields NaN instead of mixing in what the scratch held before
        if (tid == 0) atomicOr(&g_conv_status, 1u);
        for (int i = tid; i < 9 * CY * CX + CY; i += (int)blockDim.x)
            out[i] = __int_as_float(0x7fc00000);
    } else {
        const int r = warp * 32 + lane;
        for (int t = 0; t < NT; ++t) {
            float acc[CY];
            __syncwarp();
#pragma unroll
            for (int h = 0; h < CY / 16; ++h) {
                uint32_t v[16];
                tc::tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(t * CY + 16 * h), v);
                tc::tmem_wait_ld();
#pragma unroll
                for (int j = 0; j < 16; ++j) acc[16 * h + j] = it ? __uint_as_float(v[j]) : 0.0f;
            }
            const int s = t * TPT + r / CX, ci = r % CX;
            if (s < 9) {
#pragma unroll
                for (int co = 0; co < CY; ++co) out[(s * CY + co) * CX + ci] = acc[co];
            } else if (s == 9 && ci == 0) {
#pragma unroll
                for (int co = 0; co < CY; ++co) out[9 * CY * CX + co] = acc[co];
            }
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, NCOLS);
}

// dW[co][ci][tap] = sum over CTAs of partial[cta][tap][co][ci]; db[co] likewise.
// Two levels in a fixed order: thread row j of a CTA sums the blocks
// g = j, j + 16, j + 32, ... of 32 consecutive outputs (each warp reads 128
// contiguous bytes per block), then the 16 row sums are added in row order.
// The result does not depend on scheduling.
constexpr int kRedCols = 32, kRedRows = 16;

__global__ void __launch_bounds__(kRedCols * kRedRows)
    k_wgrad_reduce(const float* __restrict__ partial, int grid, int cx, int cy,
                   float* __restrict__ dw, float* __restrict__ db) {
    __shared__ float part[kRedRows][kRedCols + 1];
    const int per = 9 * cy * cx + cy;
    const int i = (int)blockIdx.x * kRedCols + (int)threadIdx.x;
    const int j = (int)threadIdx.y;
    float s = 0.0f;
    if (i < per) {
        int g = j;
        // four independent loads in flight, summed in order
        for (; g + 3 * kRedRows < grid; g += 4 * kRedRows) {
            const float a = partial[(size_t)g * per + i];
            const float b = partial[(size_t)(g + kRedRows) * per + i];
            const float c = partial[(size_t)(g + 2 * kRedRows) * per + i];
            const float d = partial[(size_t)(g + 3 * kRedRows) * per + i];
            s = (((s + a) + b) + c) + d;
        }
        for (; g < grid; g += kRedRows) s += partial[(size_t)g * per + i];
    }
    part[j][threadIdx.x] = s;
    __syncthreads();
    if (j != 0 || i >= per) return;
    float t = part[0][threadIdx.x];
#pragma unroll
    for (int r = 1; r < kRedRows; ++r) t += part[r][threadIdx.x];
    if (i < 9 * cy * cx) {
        const int tap = i / (cy * cx), rem = i - tap * cy * cx;
        const int co = rem / cx, ci = rem - co * cx;
        dw[((size_t)co * cx + ci) * 9 + tap] = t;
    } else if (db) {
        db[i - 9 * cy * cx] = t;
    }
}

void launch_wgrad_reduce(const float* partial, int grid, int cx, int cy, float* dw, float* db,
                         cudaStream_t s) {
    const int per = 9 * cy * cx + cy;
    k_wgrad_reduce<<<(per + kRedCols - 1) / kRedCols, dim3(kRedCols, kRedRows), 0, s>>>(partial, grid, cx,
                                                                                        cy, dw, db);
}

// Packed weights from OIHW binary32 W[co][ci][3][3] (cout x cin):
//   forward  : P[tap][ci / 8][co][ci % 8] = W[co][ci][tap]
//   transpose: P[tap][co / 8][ci][co % 8] = W[co][ci][8 - tap]  (data gradient)
__global__ void k_pack_weights(const float* __restrict__ w, bf16* __restrict__ p, int cin, int cout,
                               int transpose) {
    const int n = 9 * cin * cout;
    const int i = (int)(blockIdx.x * blockDim.x + threadIdx.x);
    if (i >= n) return;
    const int ki = transpose ? cout : cin;  // K channels of the packed operand
    const int ni = transpose ? cin : cout;  // N rows
    const int j = i % 8, rest = i / 8;
    const int nrow = rest % ni, rest2 = rest / ni;
    const int kc = rest2 % (ki / 8), tap = rest2 / (ki / 8);
    const int kch = kc * 8 + j;
    float v;
    if (!transpose)
        v = w[((size_t)nrow * cin + kch) * 9 + tap];
    else
        v = w[((size_t)kch * cin + nrow) * 9 + (8 - tap)];
    p[i] = __float2bfloat16_rn(v);
}

template <int CIN, int COUT>
cudaError_t launch_fwd_ws(const ConvFwdArgs& a, cudaStream_t s, bool* used);

template <int CIN, int COUT>
cudaError_t launch_fwd(const ConvFwdArgs& a, cudaStream_t s) {
    bool used = false;
    cudaError_t e0 = launch_fwd_ws<CIN, COUT>(a, s, &used);
    if (e0 != cudaSuccess || used) return e0;
    const int smem = fwd_smem<CIN, COUT>(a.W);
    cudaError_t e = cudaFuncSetAttribute(k_conv3x3_fwd<CIN, COUT>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    k_conv3x3_fwd<CIN, COUT><<<a.B * a.tiles, kConvThreads, smem, s>>>(a);
    return cudaGetLastError();
}

// 0: one tile per CTA; 1: the persistent warp-specialised forward for the
// 32 -> 32 channel layers (the pairs where it measured faster on a B200);
// 2: the persistent forward for every built pair. Both honour the width limit.
int g_conv_pipeline = 1;

PFN_cuTensorMapEncodeTiled_v12000 encode_tiled() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

// The persistent forward; *used = false (nothing launched) when the shape or
// the driver does not allow it.
template <int CIN, int COUT>
cudaError_t launch_fwd_ws(const ConvFwdArgs& a, cudaStream_t s, bool* used) {
    *used = false;
    const int smem = ws_smem<CIN, COUT>(a.W);
    PFN_cuTensorMapEncodeTiled_v12000 encode = encode_tiled();
    if (!g_conv_pipeline || (g_conv_pipeline == 1 && !(CIN == 32 && COUT == 32)) || !encode ||
        ws_box(a.W) > 256 || smem > 227 * 1024)
        return cudaSuccess;
    const int P2 = (a.H + 2) * (a.W + 2);
    // activations [B][P2][CIN] as 8 channels x CIN/8 chunks x P2 positions x B images
    const cuuint64_t dims[4] = {8, (cuuint64_t)(CIN / 8), (cuuint64_t)P2, (cuuint64_t)a.B};
    const cuuint64_t strides[3] = {16, (cuuint64_t)CIN * 2, (cuuint64_t)P2 * CIN * 2};
    const cuuint32_t box[4] = {8, 1, (cuuint32_t)ws_box(a.W), 1};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    CUtensorMap map;
    if (encode(&map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<bf16*>(a.x), dims, strides, box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return cudaSuccess;
    cudaError_t e = cudaFuncSetAttribute(k_conv3x3_fwd_ws<CIN, COUT>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    int per = 0, dev = 0, sms = 0;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_conv3x3_fwd_ws<CIN, COUT>, kWsThreads,
                                                           smem)) != cudaSuccess ||
        (e = cudaGetDevice(&dev)) != cudaSuccess ||
        (e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess)
        return e;
    // every resident CTA must get its TMEM columns (512 per SM)
    const int cols = 2 * (int)fwd_tmem_cols<COUT>();
    per = per < 512 / cols ? per : 512 / cols;
    if (per < 1) return cudaSuccess;
    const int items = a.B * a.tiles;
    const int grid = items < sms * per ? items : sms * per;
    k_conv3x3_fwd_ws<CIN, COUT><<<grid, kWsThreads, smem, s>>>(a, map);
    *used = true;
    return cudaGetLastError();
}

template <int CX, int CY>
cudaError_t launch_wgrad(const ConvWgradArgs& a, cudaStream_t s) {
    constexpr int smem = wg_smem<CX, CY>();
    cudaError_t e = cudaFuncSetAttribute(k_conv3x3_wgrad<CX, CY>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    k_conv3x3_wgrad<CX, CY><<<a.B * a.ctas, kConvThreads, smem, s>>>(a);
    return cudaGetLastError();
}

bool shape_ok(int B, int H, int W) {
    return B > 0 && H >= 2 && W >= 2 && H <= 1024 && W <= 1024 && fwd_smem<32, 64>(W) <= 227 * 1024;
}

}  // namespace

// ---- internal entry points ------------------------------------------------------

int conv3x3_fwd(const void* x, void* y, float* yf, const void* wp, const float* bias,
                const void* gate, int B, int H, int W, int cin, int cout, int relu,
                cudaStream_t s) {
    if (!x || !wp || (!y && !yf)) return set_error(PFB_E_ARG, "conv3x3: null buffer");
    if (!shape_ok(B, H, W)) return set_error(PFB_E_ARG, "conv3x3: bad shape %dx%dx%d", B, H, W);
    if ((uintptr_t)x % 16 || (uintptr_t)wp % 16 || (y && (uintptr_t)y % 16) ||
        (yf && (uintptr_t)yf % 16) || (gate && (uintptr_t)gate % 16))
        return set_error(PFB_E_ARG, "conv3x3: buffers must be 16-byte aligned");
    ConvFwdArgs a;
    a.x = static_cast<const bf16*>(x);
    a.y = static_cast<bf16*>(y);
    a.yf = yf;
    a.w = static_cast<const bf16*>(wp);
    a.bias = bias;
    a.gate = static_cast<const bf16*>(gate);
    a.B = B;
    a.H = H;
    a.W = W;
    a.relu = relu ? 1 : 0;
    a.tiles = (H * (W + 2) + kConvMT * 128 - 1) / (kConvMT * 128);
    cudaError_t e;
    if (cin == 16 && cout == 32)
        e = launch_fwd<16, 32>(a, s);
    else if (cin == 32 && cout == 32)
        e = launch_fwd<32, 32>(a, s);
    else if (cin == 32 && cout == 16)
        e = launch_fwd<32, 16>(a, s);
    else if (cin == 16 && cout == 16)
        e = launch_fwd<16, 16>(a, s);
    else
        return set_error(PFB_E_CONFIG, "conv3x3: channels %d -> %d not built", cin, cout);
    if (e != cudaSuccess) return set_error(PFB_E_CUDA, "conv3x3: %s", cudaGetErrorString(e));
    return PFB_OK;
}

size_t conv3x3_wgrad_workspace(int B, int H, int W, int cx, int cy) {
    const int total = (H * (W + 2) + kWgKT - 1) / kWgKT;
    const int ctas = total < 8 ? 1 : 2;
    return (size_t)B * ctas * (size_t)(9 * cy * cx + cy) * sizeof(float);
}

int conv3x3_wgrad(const void* x, const void* dy, float* workspace, size_t workspace_bytes,
                  float* dw, float* db, int B, int H, int W, int cx, int cy, cudaStream_t s) {
    if (!x || !dy || !workspace || !dw) return set_error(PFB_E_ARG, "conv3x3_wgrad: null buffer");
    if (!shape_ok(B, H, W)) return set_error(PFB_E_ARG, "conv3x3_wgrad: bad shape");
    if ((uintptr_t)x % 16 || (uintptr_t)dy % 16)
        return set_error(PFB_E_ARG, "conv3x3_wgrad: buffers must be 16-byte aligned");
    if (workspace_bytes < conv3x3_wgrad_workspace(B, H, W, cx, cy))
        return set_error(PFB_E_ARG, "conv3x3_wgrad: workspace too small");
    const int total = (H * (W + 2) + kWgKT - 1) / kWgKT;
    ConvWgradArgs a;
    a.x = static_cast<const bf16*>(x);
    a.dy = static_cast<const bf16*>(dy);
    a.partial = workspace;
    a.B = B;
    a.H = H;
    a.W = W;
    a.ctas = total < 8 ? 1 : 2;
    a.chunks = (total + a.ctas - 1) / a.ctas;
    cudaError_t e;
    if (cx == 16 && cy == 32)
        e = launch_wgrad<16, 32>(a, s);
    else if (cx == 32 && cy == 32)
        e = launch_wgrad<32, 32>(a, s);
    else if (cx == 32 && cy == 16)
        e = launch_wgrad<32, 16>(a, s);
    else if (cx == 16 && cy == 16)
        e = launch_wgrad<16, 16>(a, s);
    else
        return set_error(PFB_E_CONFIG, "conv3x3_wgrad: channels %d, %d not built", cx, cy);
    if (e != cudaSuccess) return set_error(PFB_E_CUDA, "conv3x3_wgrad: %s", cudaGetErrorString(e));
    launch_wgrad_reduce(workspace, B * a.ctas, cx, cy, dw, db, s);
    e = cudaGetLastError();
    if (e != cudaSuccess) return set_error(PFB_E_CUDA, "wgrad reduce: %s", cudaGetErrorString(e));
    return PFB_OK;
}

int conv3x3_pack(const float* w, void* packed, int cin, int cout, int transpose, cudaStream_t s) {
    if (!w || !packed) return set_error(PFB_E_ARG, "conv3x3_pack: null buffer");
    if (cin % 8 || cout % 8 || cin <= 0 || cout <= 0)
        return set_error(PFB_E_ARG, "conv3x3_pack: channels must be multiples of 8");
    const int n = 9 * cin * cout;
    k_pack_weights<<<(n + 255) / 256, 256, 0, s>>>(w, static_cast<bf16*>(packed), cin, cout,
                                                    transpose ? 1 : 0);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return set_error(PFB_E_CUDA, "conv3x3_pack: %s", cudaGetErrorString(e));
    return PFB_OK;
}

int conv_read_status(unsigned* out, int clear) {
    unsigned v = 0;
    cudaError_t e = cudaMemcpyFromSymbol(&v, g_conv_status, sizeof(v));
    if (e != cudaSuccess) return set_error(PFB_E_CUDA, "conv status: %s", cudaGetErrorString(e));
    if (clear) {
        const unsigned z = 0;
        e = cudaMemcpyToSymbol(g_conv_status, &z, sizeof(z));
        if (e != cudaSuccess) return set_error(PFB_E_CUDA, "conv status: %s", cudaGetErrorString(e));
    }
    if (out) *out = v;
    return PFB_OK;
}

}  // namespace pfb

// ---- C ABI (include/pfb200_surrogate.h) ----------------------------------------

extern "C" {

int pfb_conv3x3_forward(const void* x, void* y, float* y_f32, const void* w_packed,
                        const float* bias, const void* gate, int batch, int H, int W, int cin,
                        int cout, int relu, void* stream) {
    pfb::clear_error();
    return pfb::conv3x3_fwd(x, y, y_f32, w_packed, bias, gate, batch, H, W, cin, cout, relu,
                            static_cast<cudaStream_t>(stream));
}

int pfb_conv3x3_pack(const float* w_oihw, void* w_packed, int cin, int cout, int transpose,
                     void* stream) {
    pfb::clear_error();
    return pfb::conv3x3_pack(w_oihw, w_packed, cin, cout, transpose,
                             static_cast<cudaStream_t>(stream));
}

size_t pfb_conv3x3_wgrad_workspace(int batch, int H, int W, int cx, int cy) {
    return pfb::conv3x3_wgrad_workspace(batch, H, W, cx, cy);
}

int pfb_conv3x3_wgrad(const void* x, const void* dy, float* workspace, size_t workspace_bytes,
                      float* dw_oihw, float* db, int batch, int H, int W, int cx, int cy,
                      void* stream) {
    pfb::clear_error();
    return pfb::conv3x3_wgrad(x, dy, workspace, workspace_bytes, dw_oihw, db, batch, H, W, cx, cy,
                              static_cast<cudaStream_t>(stream));
}

int pfb_conv_status(unsigned* out, int clear) { return pfb::conv_read_status(out, clear); }

int pfb_conv_set_pipeline(int mode) {
    pfb::clear_error();
    if (mode < 0 || mode > 2) return pfb::set_error(PFB_E_ARG, "conv pipeline mode %d not in 0..2", mode);
    pfb::g_conv_pipeline = mode;
    return PFB_OK;
}

}  // extern "C"

// ---- weight gradient without caller workspace -----------------------------------
//
// Some callers cannot hand this library device memory for scratch: hosts
// whose device memory is owned by their own pool allocator (a training
// framework's caching allocator, a serving engine's preallocated arena) and
// that forbid a raw cudaMalloc, which would take memory outside their budget
// and, being synchronizing, stall their streams. For them the weight gradient
// keeps its partial sums in this fixed array instead, which every GPU that
// loads the library holds until the process exits. Calls that overlap on the
// GPU (two streams, or two host threads) share the array and race.

using namespace pfb;

namespace {

constexpr size_t kNoAllocScratchBytes = (size_t)4 << 20;  // 4 MiB per device
constexpr int kNoAllocMaxDevices = 64;

static __device__ __align__(256) float g_wgrad_scratch[kNoAllocScratchBytes / sizeof(float)];

std::mutex g_scratch_mutex;
float* g_scratch_ptr[kNoAllocMaxDevices] = {};

// Device address of g_wgrad_scratch on the current device, looked up once per
// device (the host-side name of the array is not a device address). The
// address belongs to the device's primary context: a cudaDeviceReset in the
// same process makes the cached value stale, so such hosts must not call the
// entry point after a reset.
int scratch_on_current_device(float** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return set_error(PFB_E_CUDA, "cudaGetDevice: %s", cudaGetErrorString(e));
    if (dev < 0 || dev >= kNoAllocMaxDevices)
        return set_error(PFB_E_CONFIG, "device %d beyond the %d supported", dev, kNoAllocMaxDevices);
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!g_scratch_ptr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_wgrad_scratch);
        if (e != cudaSuccess || !p)
            return set_error(PFB_E_CUDA, "scratch address: %s", cudaGetErrorString(e));
        g_scratch_ptr[dev] = static_cast<float*>(p);
    }
    *out = g_scratch_ptr[dev];
    return PFB_OK;
}

}  // namespace

extern "C" int pfb_conv3x3_wgrad_noalloc(const void* x, const void* dy, float* dw_oihw, float* db,
                                         int batch, int H, int W, int cx, int cy, void* stream) {
    clear_error();
    if (!x || !dy || !dw_oihw) return set_error(PFB_E_ARG, "conv3x3_wgrad_noalloc: null buffer");
    if (!shape_ok(batch, H, W))
        return set_error(PFB_E_ARG, "conv3x3_wgrad_noalloc: bad shape %dx%dx%d", batch, H, W);
    if (cx <= 0 || cy <= 0 || cx > 64 || cy > 64)
        return set_error(PFB_E_CONFIG, "conv3x3_wgrad_noalloc: channels %d, %d not built", cx, cy);
    const size_t need = conv3x3_wgrad_workspace(batch, H, W, cx, cy);
    if (need > kNoAllocScratchBytes)
        return set_error(PFB_E_ARG,
                         "conv3x3_wgrad_noalloc: %d images of %dx%d with %d -> %d channels need "
                         "%zu bytes of scratch, above its fixed %zu bytes (split the batch, or "
                         "use pfb_conv3x3_wgrad with a workspace)",
                         batch, H, W, cx, cy, need, kNoAllocScratchBytes);
    float* scratch = nullptr;
    const int rc = scratch_on_current_device(&scratch);
    if (rc) return rc;
    // every CTA overwrites its whole block of partial sums before the reduction
    // reads it (with NaN when its MMA wait gave up), so nothing in the shared
    // array has to start at zero
    return conv3x3_wgrad(x, dy, scratch, kNoAllocScratchBytes, dw_oihw, db, batch, H, W, cx, cy,
                         static_cast<cudaStream_t>(stream));
}
