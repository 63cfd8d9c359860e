// PFB boundary recorder of the 2D system: compact half-height snapshots
// (reference src/boundary.cu, include/boundary.cuh, common/boundary_format.h).
//
// A frame holds, per cell, a 40-byte record (id, tile origin, periodic
// centroid, gamma, mobility, active speed, target radius, square count) and
// then every 2x2 square of its 288^2 tile whose four corner samples straddle
// phi = 1/2, with the corners kept as binary32 (lower left, lower right,
// upper right, upper left) and the square's tile position packed as x | y<<16.
// Contours are interpolated offline. Frames are framed independently (magic,
// step, time, byte counts, FNV-1a 64 of the payload); the file ends with an
// end record carrying the frame count.
//
// Squares are written in ascending tile order (row-major over the 287 x 287
// squares) within each cell; the reference's gather appends them in warp
// arrival order, so the two files hold the same squares per cell but not
// necessarily in the same order. File writes run on a background thread with
// at most three frames queued, so the simulation continues while a frame is
// written.
#include <cuda_runtime.h>

#include <cerrno>
#include <cmath>
#include <condition_variable>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "device_util.cuh"
#include "pfb200_ckpt.h"
#include "pfb_common.cuh"
#include "pfb_internal.h"

namespace pfb {
namespace {

constexpr int kBndThreads = 256;
constexpr int kSquaresPerRow = kTilePitch - 1;
constexpr int kSquares = kSquaresPerRow * kSquaresPerRow;

#pragma pack(push, 1)
struct BndCell {
    int32_t id, origin_x, origin_y;
    float cx, cy, gamma, mobility, active_speed, radius;
    uint32_t squares;
};
struct BndSquare {
    uint32_t xy;
    float phi[4];
};
struct BndFileHeader {
    char magic[8];
    uint32_t version, header_bytes, cells, side, tile_pitch, square_bytes;
    double dt, tau, level;
    uint64_t interval;
    uint32_t codec, reserved;
};
struct BndFrameHeader {
    char magic[8];
    uint64_t step;
    double time;
    uint64_t raw_bytes, stored_bytes, checksum;
};
#pragma pack(pop)
static_assert(sizeof(BndCell) == 40 && sizeof(BndSquare) == 20, "PFB records");
static_assert(sizeof(BndFileHeader) == 72 && sizeof(BndFrameHeader) == 48, "PFB headers");

// Square q of a tile: its corners and whether phi = 1/2 separates them.
__device__ __forceinline__ bool square_at(const float* tile, int q, BndSquare* s) {
    const int x = q % kSquaresPerRow, y = q / kSquaresPerRow;
    const int j = y * kTilePitch + x;
    s->xy = (uint32_t)x | ((uint32_t)y << 16);
    s->phi[0] = tile[j];
    s->phi[1] = tile[j + 1];
    s->phi[2] = tile[j + kTilePitch + 1];
    s->phi[3] = tile[j + kTilePitch];
    const bool in = s->phi[0] >= 0.5f;
    return (s->phi[1] >= 0.5f) != in || (s->phi[2] >= 0.5f) != in || (s->phi[3] >= 0.5f) != in;
}

// One CTA per cell: count the crossed squares, flag a non-finite sample
// (count UINT32_MAX), and fill the cell record.
__global__ void __launch_bounds__(kBndThreads)
    k_bnd_count(const float* phi, const pfb_cell2d* cells, BndCell* meta, int side) {
    const int i = blockIdx.x, t = threadIdx.x;
    const float* tile = phi + (size_t)i * kTileArea;
    unsigned count = 0, bad = 0;
    for (int q = t; q < kSquares; q += kBndThreads) {
        BndSquare s;
        count += square_at(tile, q, &s) ? 1u : 0u;
        for (int k = 0; k < 4; ++k) bad |= isfinite(s.phi[k]) ? 0u : 1u;
    }
    count = __reduce_add_sync(0xFFFFFFFFu, count);
    bad = __reduce_or_sync(0xFFFFFFFFu, bad);
    __shared__ unsigned wc[kBndThreads / 32], wb[kBndThreads / 32];
    if ((t & 31) == 0) {
        wc[t >> 5] = count;
        wb[t >> 5] = bad;
    }
    __syncthreads();
    if (t == 0) {
        unsigned total = 0, invalid = 0;
        for (int w = 0; w < kBndThreads / 32; ++w) {
            total += wc[w];
            invalid |= wb[w];
        }
        const pfb_cell2d c = cells[i];
        const Window win = window_of(c.cls);
        BndCell m;
        m.id = c.global_id;
        m.origin_x = ((c.gx0 - win.tx0) % side + side) % side;
        m.origin_y = ((c.gy0 - win.ty0) % side + side) % side;
        const double x = (double)c.gx0 + c.Cx / c.V;
        const double y = (double)c.gy0 + c.Cy / c.V;
        m.cx = (float)(x - floor(x / side) * side);
        m.cy = (float)(y - floor(y / side) * side);
        m.gamma = c.gamma;
        m.mobility = c.M_pf;
        m.active_speed = c.v_A;
        m.radius = c.R_tgt;
        m.squares = invalid ? 0xFFFFFFFFu : total;
        meta[i] = m;
    }
}

// One CTA per cell: the crossed squares in ascending tile order from
// out[offsets[i]] (a block-wide exclusive scan per chunk of 256 squares).
__global__ void __launch_bounds__(kBndThreads)
    k_bnd_gather(const float* phi, const uint64_t* offsets, BndSquare* out) {
    const int i = blockIdx.x, t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const float* tile = phi + (size_t)i * kTileArea;
    __shared__ unsigned wsum[kBndThreads / 32];
    BndSquare* dst = out + offsets[i];
    unsigned base = 0;
    for (int q0 = 0; q0 < kSquares; q0 += kBndThreads) {
        const int q = q0 + t;
        BndSquare s;
        const bool hit = q < kSquares && square_at(tile, q, &s);
        const unsigned mask = __ballot_sync(0xFFFFFFFFu, hit);
        if (lane == 0) wsum[warp] = __popc(mask);
        __syncthreads();
        unsigned before = 0, total = 0;
        for (int w = 0; w < kBndThreads / 32; ++w) {
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

}  // namespace

struct Boundary2D {
    std::FILE* f = nullptr;
    int N = 0, side = 0;
    BndCell* d_meta = nullptr;
    uint64_t* d_off = nullptr;
    BndSquare* d_sq = nullptr;
    size_t capacity = 0;
    std::vector<BndCell> meta;
    std::vector<uint64_t> off;
    // writer thread and its queue of finished frames
    struct Frame {
        std::vector<unsigned char> data;
        uint64_t step;
        double time;
    };
    std::deque<Frame> queue;
    std::mutex mu;
    std::condition_variable cv;
    std::thread worker;
    bool stopping = false, failed = false, capture_failed = false;
    uint64_t frames = 0, last_step = 0;
    double last_time = 0.0;

    ~Boundary2D() {
        if (worker.joinable()) finish();
        if (f) std::fclose(f);
        cudaFree(d_meta);
        cudaFree(d_off);
        cudaFree(d_sq);
    }

    bool put(const void* p, size_t n) { return std::fwrite(p, 1, n, f) == n; }

    void write_loop() {
        for (;;) {
            Frame fr;
            {
                std::unique_lock<std::mutex> lock(mu);
                cv.wait(lock, [&] { return stopping || !queue.empty(); });
                if (queue.empty()) return;
                fr = std::move(queue.front());
                queue.pop_front();
            }
            BndFrameHeader h{};
            std::memcpy(h.magic, "PFBFRM1", 8);
            h.step = fr.step;
            h.time = fr.time;
            h.raw_bytes = h.stored_bytes = fr.data.size();
            h.checksum = fnv1a64(fr.data.data(), fr.data.size());
            const bool ok = put(&h, sizeof(h)) && put(fr.data.data(), fr.data.size());
            {
                std::lock_guard<std::mutex> lock(mu);
                if (!ok) {
                    failed = true;
                    queue.clear();
                } else {
                    ++frames;
                    last_step = fr.step;
                    last_time = fr.time;
                }
            }
            cv.notify_all();
            if (!ok) return;
        }
    }

    int finish() {
        {
            std::lock_guard<std::mutex> lock(mu);
            stopping = true;
        }
        cv.notify_all();
        if (worker.joinable()) worker.join();
        bool ok = !failed && !capture_failed;
        if (f) {
            if (ok) {
                BndFrameHeader end{};
                std::memcpy(end.magic, "PFBEND1", 8);
                end.step = last_step;
                end.time = last_time;
                end.checksum = frames;
                ok = put(&end, sizeof(end));
            }
            if (std::fclose(f) != 0) ok = false;
            f = nullptr;
        }
        failed = !ok;
        return ok ? PFB_OK : set_error(PFB_E_IO, "boundary: the file is incomplete");
    }

    int capture(const float* phi, const pfb_cell2d* cells, cudaStream_t stream, long long step,
                double time) {
        k_bnd_count<<<N, kBndThreads, 0, stream>>>(phi, cells, d_meta, side);
        cudaError_t e = cudaGetLastError();
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(meta.data(), d_meta, (size_t)N * sizeof(BndCell),
                                cudaMemcpyDeviceToHost, stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) return set_error(PFB_E_CUDA, "boundary count: %s", cudaGetErrorString(e));
        uint64_t total = 0;
        for (int i = 0; i < N; ++i) {
            if (meta[(size_t)i].squares == 0 || meta[(size_t)i].squares == 0xFFFFFFFFu)
                return set_error(PFB_E_STATE, "boundary: cell %d has a missing or non-finite boundary",
                                 meta[(size_t)i].id);
            off[(size_t)i] = total;
            total += meta[(size_t)i].squares;
        }
        const size_t prefix = (size_t)N * sizeof(BndCell);
        const uint64_t bytes = prefix + total * sizeof(BndSquare);
        if (bytes > (1ull << 31)) return set_error(PFB_E_STATE, "boundary: frame exceeds 2 GiB");
        if (total > capacity) {
            cudaFree(d_sq);
            d_sq = nullptr;
            capacity = (size_t)(total + total / 8 + 256);
            if ((e = cudaMalloc(&d_sq, capacity * sizeof(BndSquare))) != cudaSuccess)
                return set_error(PFB_E_CUDA, "boundary: %s", cudaGetErrorString(e));
        }
        if ((e = cudaMemcpyAsync(d_off, off.data(), (size_t)N * sizeof(uint64_t),
                                 cudaMemcpyHostToDevice, stream)) != cudaSuccess)
            return set_error(PFB_E_CUDA, "boundary: %s", cudaGetErrorString(e));
        k_bnd_gather<<<N, kBndThreads, 0, stream>>>(phi, d_off, d_sq);
        if ((e = cudaGetLastError()) != cudaSuccess)
            return set_error(PFB_E_CUDA, "boundary gather: %s", cudaGetErrorString(e));
        Frame fr;
        fr.step = (uint64_t)step;
        fr.time = time;
        fr.data.resize((size_t)bytes);
        std::memcpy(fr.data.data(), meta.data(), prefix);
        if ((e = cudaMemcpyAsync(fr.data.data() + prefix, d_sq, (size_t)total * sizeof(BndSquare),
                                 cudaMemcpyDeviceToHost, stream)) != cudaSuccess ||
            (e = cudaStreamSynchronize(stream)) != cudaSuccess)
            return set_error(PFB_E_CUDA, "boundary readback: %s", cudaGetErrorString(e));
        {
            std::unique_lock<std::mutex> lock(mu);
            cv.wait(lock, [&] { return failed || queue.size() < 3; });
            if (failed) return set_error(PFB_E_IO, "boundary: write failed");
            queue.push_back(std::move(fr));
        }
        cv.notify_all();
        return PFB_OK;
    }
};

Boundary2D* boundary2d_open(const char* path, int N, int side, double dt, double tau,
                            long long interval, int compress) {
    if (!path || !path[0] || N <= 0 || side <= 0 || interval <= 0 || !std::isfinite(dt) ||
        dt <= 0.0 || !std::isfinite(tau) || tau <= 0.0) {
        set_error(PFB_E_ARG, "boundary: invalid output geometry or cadence");
        return nullptr;
    }
    if (compress) {
        set_error(PFB_E_CONFIG, "boundary: this build has no zstd; select --boundary-compression none");
        return nullptr;
    }
    Boundary2D* b = new Boundary2D();
    b->N = N;
    b->side = side;
    b->meta.resize((size_t)N);
    b->off.resize((size_t)N);
    if (cudaMalloc(&b->d_meta, (size_t)N * sizeof(BndCell)) != cudaSuccess ||
        cudaMalloc(&b->d_off, (size_t)N * sizeof(uint64_t)) != cudaSuccess) {
        delete b;
        set_error(PFB_E_CUDA, "boundary: allocation failed");
        return nullptr;
    }
    b->f = std::fopen(path, "wbx");  // a new file only
    if (!b->f) {
        set_error(PFB_E_IO, "boundary: cannot create new output file %s: %s", path, std::strerror(errno));
        delete b;
        return nullptr;
    }
    BndFileHeader h{};
    std::memcpy(h.magic, "PFBND01", 8);
    h.version = 1;
    h.header_bytes = sizeof(h);
    h.cells = (uint32_t)N;
    h.side = (uint32_t)side;
    h.tile_pitch = kTilePitch;
    h.square_bytes = sizeof(BndSquare);
    h.dt = dt;
    h.tau = tau;
    h.level = 0.5;
    h.interval = (uint64_t)interval;
    h.codec = 0;
    if (!b->put(&h, sizeof(h))) {
        set_error(PFB_E_IO, "boundary: header write failed");
        delete b;
        return nullptr;
    }
    b->worker = std::thread([b] { b->write_loop(); });
    return b;
}

int boundary2d_capture(Boundary2D* b, const float* phi, const pfb_cell2d* cells,
                       cudaStream_t stream, long long step, double time) {
    const int rc = b->capture(phi, cells, stream, step, time);
    if (rc) b->capture_failed = true;
    return rc;
}

int boundary2d_close(Boundary2D* b) {
    const int rc = b->finish();
    delete b;
    return rc;
}

}  // namespace pfb
