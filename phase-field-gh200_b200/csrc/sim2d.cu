// Host driver of the 2D update (the reference's `Sim`, include/sim.cuh:58-152
// and src/sim.cu:159-1055) and the C-ABI wrappers of the 2D kernels.
//
// Buffer scheme kept from the reference so slots, parities and graph replay
// line up with it: two phi pools (parity = step % 2), three S slots (read
// step % 3, scatter (step+1) % 3, clear (step+2) % 3), device-resident step
// counters and cursors in two slots following the phi parity, and a captured
// CUDA graph of six steps that covers every (parity, slot) pair.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <vector>

#include "pfb_common.cuh"
#include "pfb_internal.h"

using namespace pfb;

#define PFB_CU(expr, what)                                                              \
    do {                                                                                \
        const cudaError_t e_ = (expr);                                                  \
        if (e_ != cudaSuccess) return set_error(PFB_E_CUDA, "%s: %s", what, cudaGetErrorString(e_)); \
    } while (0)

struct pfb_sim2d {
    pfb_params2d p{};
    int device = 0;
    int L = 0, P = 0, N = 0;
    size_t s_words = 0;
    float* d_phi[2] = {nullptr, nullptr};
    uint32_t* d_S = nullptr;
    pfb_cell2d* d_cell = nullptr;
    pfb_cell2d* d_cell_prev = nullptr;  // records before the last residual step
    // in-memory device checkpoint (pfb_sim2d_save / pfb_sim2d_restore)
    void* b_phi = nullptr;
    pfb_cell2d* b_cell = nullptr;
    uint8_t* b_cls = nullptr;
    uint32_t* b_S = nullptr;
    uint32_t* b_flags = nullptr;
    long long b_step = -1;
    uint8_t* d_cls = nullptr;
    unsigned long long* d_cursor = nullptr;
    unsigned long long* d_step = nullptr;
    uint32_t* d_flags = nullptr;
    pfb_traj_cell2d* d_traj = nullptr;
    cudaStream_t stream = nullptr;
    long long steps_done = 0;
    int cluster = kDefaultCluster;
    int variant = 0;
    bool use_graph = true;
    bool graph_ready = false;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    // six-step graphs that also pack a trajectory frame into the host ring
    // after every `every`-th step, [every - 1][phase] for every = 1, 2, 3, 6
    // and the call's step count modulo `every` at the graph's start
    cudaGraphExec_t rec_exec[6][6] = {};
    TrajRing2D* d_ring = nullptr;
    Velocity2D* vel = nullptr;  // open PFVMOM4 recorder
    Boundary2D* bnd = nullptr;  // open PFB recorder
    uint32_t* d_perm = nullptr;  // Morton visit order (null: launch order)
    // exact overflow detection of the non-returning scatter (BinArgs)
    unsigned long long* d_bins = nullptr;
    int4* d_geo = nullptr;             // 2 x N committed window geometries
    unsigned int* d_recounts = nullptr;
    int nbins_side = 0;
    bool bins_pending = false;  // the last launch's bounds are not settled yet

    size_t bin_words() const { return 2 * (size_t)nbins_side * (size_t)nbins_side; }

    BinArgs bin_args() const {
        return BinArgs{d_bins, d_geo, d_recounts, nbins_side, nbins_side};
    }

    // Both bound sets back to zero: after any change of the step counter
    // other than a launch.
    int reset_bins() {
        PFB_CU(cudaMemsetAsync(d_bins, 0, bin_words() * sizeof(unsigned long long), stream),
               "clear bins");
        bins_pending = false;
        return PFB_OK;
    }

    // Settle the bounds of the last launch (its field is the current pool).
    int settle_bins() {
        if (!bins_pending) return PFB_OK;
        bins_pending = false;
        return step2d_settle_bins(bin_args(), d_phi[steps_done % 2], p.phi_storage, N, L,
                                  (unsigned long long)(steps_done - 1), d_flags, stream);
    }

    ~pfb_sim2d() {
        if (vel) velocity2d_destroy(vel);
        if (bnd) (void)boundary2d_close(bnd);
        if (graph_exec) cudaGraphExecDestroy(graph_exec);
        if (graph) cudaGraphDestroy(graph);
        for (auto& row : rec_exec)
            for (cudaGraphExec_t& e : row)
                if (e) cudaGraphExecDestroy(e);
        if (stream) cudaStreamDestroy(stream);
        cudaFree(d_phi[0]);
        cudaFree(d_phi[1]);
        cudaFree(d_S);
        cudaFree(d_cell);
        cudaFree(d_cls);
        cudaFree(d_cursor);
        cudaFree(d_step);
        cudaFree(d_flags);
        cudaFree(d_traj);
        cudaFree(d_ring);
        cudaFree(d_perm);
        cudaFree(d_cell_prev);
        cudaFree(d_bins);
        cudaFree(d_geo);
        cudaFree(d_recounts);
        cudaFree(b_phi);
        cudaFree(b_cell);
        cudaFree(b_cls);
        cudaFree(b_S);
        cudaFree(b_flags);
    }

    int save() {
        PFB_CU(cudaSetDevice(device), "cudaSetDevice");
        if (!b_phi) {
            PFB_CU(cudaMalloc(&b_phi, pool_bytes()), "alloc checkpoint");
            PFB_CU(cudaMalloc(&b_cell, (size_t)N * sizeof(pfb_cell2d)), "alloc checkpoint");
            PFB_CU(cudaMalloc(&b_cls, (size_t)N), "alloc checkpoint");
            PFB_CU(cudaMalloc(&b_S, s_words * sizeof(uint32_t)), "alloc checkpoint");
            PFB_CU(cudaMalloc(&b_flags, PFB_FLAG_COUNT * sizeof(uint32_t)), "alloc checkpoint");
        }
        const int pin = (int)(steps_done % 2), rot = (int)(steps_done % 3);
        PFB_CU(cudaMemcpyAsync(b_phi, d_phi[pin], pool_bytes(), cudaMemcpyDeviceToDevice, stream), "save");
        PFB_CU(cudaMemcpyAsync(b_cell, d_cell, (size_t)N * sizeof(pfb_cell2d), cudaMemcpyDeviceToDevice,
                               stream), "save");
        PFB_CU(cudaMemcpyAsync(b_cls, d_cls, (size_t)N, cudaMemcpyDeviceToDevice, stream), "save");
        PFB_CU(cudaMemcpyAsync(b_S, d_S + (size_t)rot * s_words, s_words * sizeof(uint32_t),
                               cudaMemcpyDeviceToDevice, stream), "save");
        PFB_CU(cudaMemcpyAsync(b_flags, d_flags, PFB_FLAG_COUNT * sizeof(uint32_t),
                               cudaMemcpyDeviceToDevice, stream), "save");
        b_step = steps_done;
        return PFB_OK;
    }

    // Back to the saved state: pool, cells, the aggregate slot and flags, with
    // the step counters, cursors and the other aggregate slots as a fresh
    // set_state leaves them.
    int restore() {
        if (b_step < 0) return set_error(PFB_E_STATE, "restore: nothing saved");
        PFB_CU(cudaSetDevice(device), "cudaSetDevice");
        drop_graph();
        steps_done = b_step;
        const int pin = (int)(steps_done % 2), rot = (int)(steps_done % 3);
        PFB_CU(cudaMemcpyAsync(d_phi[pin], b_phi, pool_bytes(), cudaMemcpyDeviceToDevice, stream),
               "restore");
        PFB_CU(cudaMemcpyAsync(d_cell, b_cell, (size_t)N * sizeof(pfb_cell2d), cudaMemcpyDeviceToDevice,
                               stream), "restore");
        PFB_CU(cudaMemcpyAsync(d_cls, b_cls, (size_t)N, cudaMemcpyDeviceToDevice, stream), "restore");
        PFB_CU(cudaMemsetAsync(d_S, 0, 3 * s_words * sizeof(uint32_t), stream), "restore");
        PFB_CU(cudaMemcpyAsync(d_S + (size_t)rot * s_words, b_S, s_words * sizeof(uint32_t),
                               cudaMemcpyDeviceToDevice, stream), "restore");
        PFB_CU(cudaMemcpyAsync(d_flags, b_flags, PFB_FLAG_COUNT * sizeof(uint32_t),
                               cudaMemcpyDeviceToDevice, stream), "restore");
        const unsigned long long hs[2] = {
            (unsigned long long)(pin == 0 ? steps_done : steps_done + 1),
            (unsigned long long)(pin == 1 ? steps_done : steps_done + 1)};
        PFB_CU(cudaMemcpyAsync(d_step, hs, sizeof(hs), cudaMemcpyHostToDevice, stream), "restore");
        PFB_CU(cudaMemsetAsync(d_cursor, 0, 2 * sizeof(unsigned long long), stream), "restore");
        if (const int rc = reset_bins()) return rc;
        PFB_CU(cudaStreamSynchronize(stream), "restore");
        return PFB_OK;
    }

    pfb_step_args2d args_for_slot(int slot) const {
        const int pin = slot % 2, pout = 1 - pin, rs = slot % 3;
        pfb_step_args2d a;
        std::memset(&a, 0, sizeof(a));
        pfb_fill_coefficients2d(&p, &a);
        a.phi_in = d_phi[pin];
        a.phi_out = d_phi[pout];
        a.S_rd = d_S + (size_t)rs * s_words;
        a.S_sc = d_S + (size_t)((rs + 1) % 3) * s_words;
        a.S_cl = d_S + (size_t)((rs + 2) % 3) * s_words;
        a.cell = d_cell;
        a.cell_cls = d_cls;
        a.perm = d_perm;
        a.cursor_use = d_cursor + pin;
        a.cursor_clear = d_cursor + pout;
        a.step_rd = d_step + pin;
        a.step_wr = d_step + pout;
        a.flags = d_flags;
        a.moments = nullptr;
        a.N = N;
        a.L = L;
        a.P = P;
        a.parity_out = pout;
        a.clear_ahead_words = (unsigned long long)s_words;
        return a;
    }

    // Re-sort the visit order on the first slot of every six (reference
    // src/sim.cu:649-653).
    int sort_visit_order(int slot) {
        if (d_perm && slot % 6 == 0) PFB_CU(visit_order2d_launch(d_cell, d_perm, N, L, stream), "visit order");
        return PFB_OK;
    }

    int launch_one(int slot) {
        if (const int rc = sort_visit_order(slot)) return rc;
        const pfb_step_args2d a = args_for_slot(slot);
        // the driver owns bin buffers: non-returning scatter, overflow exact
        if (variant == 0 || variant == 1) {
            bins_pending = true;
            return step2d_launch_binned(&a, cluster, p.phi_storage, bin_args(), stream);
        }
        // a returning-scatter step settles nothing: settle the last binned one first
        if (const int rc = settle_bins()) return rc;
        return step2d_launch_storage(&a, cluster, 1, p.phi_storage, stream);
    }

    size_t pool_bytes() const {
        return (size_t)N * kTileArea * (p.phi_storage ? sizeof(uint16_t) : sizeof(float));
    }

    // Field of a 16-bit pool in binary32 (a temporary of N tiles).
    int widen(int pool, float* out) {
        return widen_pool(d_phi[pool], out, (size_t)N * kTileArea, p.phi_storage, stream);
    }

    void drop_graph() {
        if (graph_exec) cudaGraphExecDestroy(graph_exec);
        if (graph) cudaGraphDestroy(graph);
        graph_exec = nullptr;
        graph = nullptr;
        graph_ready = false;
        for (auto& row : rec_exec)
            for (cudaGraphExec_t& e : row) {
                if (e) cudaGraphExecDestroy(e);
                e = nullptr;
            }
    }

    // The six steps of the plain graph with a ring frame packed after local
    // step s whenever (phase + s + 1) is a multiple of `every` (every
    // divides 6, 0 <= phase < every).
    int build_record_graph(int every, int phase) {
        if (const int rc = settle_bins()) return rc;
        PFB_CU(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal), "begin capture");
        int rc = PFB_OK;
        for (int s = 0; s < 6 && rc == PFB_OK; ++s) {
            rc = launch_one(s);
            if (rc == PFB_OK && (phase + s + 1) % every == 0)
                rc = pack_traj2d_ring(d_cell, d_cls, d_ring, N, L, stream);
        }
        bins_pending = false;
        cudaGraph_t g = nullptr;
        const cudaError_t e = cudaStreamEndCapture(stream, &g);
        if (rc != PFB_OK) {
            if (g) cudaGraphDestroy(g);
            return rc;
        }
        PFB_CU(e, "end capture");
        const cudaError_t ie = cudaGraphInstantiateWithFlags(&rec_exec[every - 1][phase], g, 0);
        cudaGraphDestroy(g);
        PFB_CU(ie, "graph instantiate");
        return PFB_OK;
    }

    int build_graph() {
        drop_graph();
        if (const int rc = settle_bins()) return rc;  // capture marks nothing as run
        PFB_CU(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal), "begin capture");
        int rc = PFB_OK;
        for (int s = 0; s < 6 && rc == PFB_OK; ++s) rc = launch_one(s);
        bins_pending = false;
        cudaGraph_t g = nullptr;
        const cudaError_t e = cudaStreamEndCapture(stream, &g);
        if (rc != PFB_OK) {
            if (g) cudaGraphDestroy(g);
            return rc;
        }
        PFB_CU(e, "end capture");
        graph = g;
        PFB_CU(cudaGraphInstantiateWithFlags(&graph_exec, graph, 0), "graph instantiate");
        graph_ready = true;
        return PFB_OK;
    }

    // One observed step while a velocity recorder is open.
    int launch_observed() {
        if (const int rc = sort_visit_order((int)(steps_done % 6))) return rc;
        pfb_step_args2d a = args_for_slot((int)(steps_done % 6));
        int obs = PFB_VELOCITY_DISABLED;
        int rc = velocity2d_prepare(vel, &a, steps_done, stream, &obs);
        if (rc) return rc;
        if ((rc = step2d_launch_observed(&a, cluster, obs, stream))) return rc;
        velocity2d_advanced(vel);
        return PFB_OK;
    }

    int advance(long long steps) {
        if (vel) {
            for (; steps > 0; --steps, ++steps_done) {
                const int rc = launch_observed();
                if (rc) return rc;
            }
            return PFB_OK;
        }
        while (steps > 0) {
            if (use_graph && !graph_ready) {
                const int rc = build_graph();
                if (rc) return rc;
            }
            if (use_graph && graph_ready && steps_done % 6 == 0 && steps >= 6) {
                PFB_CU(cudaGraphLaunch(graph_exec, stream), "graph launch");
                bins_pending = variant == 0 || variant == 1;
                steps_done += 6;
                steps -= 6;
            } else {
                const int rc = launch_one((int)(steps_done % 6));
                if (rc) return rc;
                steps_done += 1;
                steps -= 1;
            }
        }
        // nothing stays pending across calls: the caller may read flags or
        // change the field next
        return settle_bins();
    }

    // `steps` steps with the trajectory records of every `every`-th step
    // written to ring frame k % frames (k = 0, 1, ... in this call), all
    // queued without a host wait. A ring in page-locked memory is written by
    // the device directly, and six-step graphs carry the records where the
    // interval divides six; any other ring gets a copy after each pack.
    // Plain six-step graphs run where no record falls inside the six steps.
    int advance_record(long long steps, int every, pfb_traj_cell2d* ring, int frames) {
        const size_t frame_bytes = (size_t)N * sizeof(pfb_traj_cell2d);
        pfb_traj_cell2d* dring = nullptr;
        cudaPointerAttributes at{};
        if (cudaPointerGetAttributes(&at, ring) == cudaSuccess && at.type == cudaMemoryTypeHost &&
            at.devicePointer && !((uintptr_t)at.devicePointer & 15u))
            dring = static_cast<pfb_traj_cell2d*>(at.devicePointer);
        (void)cudaGetLastError();  // an unregistered pointer is not an error here
        if (dring) {
            if (!d_ring) PFB_CU(cudaMalloc(&d_ring, sizeof(TrajRing2D)), "alloc ring");
            if (const int rc = ring_begin2d(d_ring, dring, frames, stream)) return rc;
        }
        const bool rec_graph = dring && !vel && use_graph && 6 % every == 0;
        long long done = 0, k = 0;
        while (done < steps) {
            const bool aligned = !vel && use_graph && steps_done % 6 == 0 && steps - done >= 6;
            if (rec_graph && aligned) {
                const int phase = (int)(done % every);
                if (!rec_exec[every - 1][phase]) {
                    if (const int rc = build_record_graph(every, phase)) return rc;
                }
                PFB_CU(cudaGraphLaunch(rec_exec[every - 1][phase], stream), "graph launch");
                bins_pending = variant == 0 || variant == 1;
                steps_done += 6;
                done += 6;
                continue;
            }
            if (!vel && use_graph && !graph_ready) {
                const int rc = build_graph();
                if (rc) return rc;
            }
            // next record after step index `due` of this call (1-based)
            const long long due = (done / every + 1) * every;
            if (aligned && graph_ready && due >= done + 6) {
                PFB_CU(cudaGraphLaunch(graph_exec, stream), "graph launch");
                bins_pending = variant == 0 || variant == 1;
                steps_done += 6;
                done += 6;
            } else {
                const int rc = vel ? launch_observed() : launch_one((int)(steps_done % 6));
                if (rc) return rc;
                steps_done += 1;
                done += 1;
            }
            if (done % every == 0) {
                if (dring) {
                    if (const int rc = pack_traj2d_ring(d_cell, d_cls, d_ring, N, L, stream)) return rc;
                } else {
                    if (const int rc = pack_traj2d(d_cell, d_cls, d_traj, N, L, stream)) return rc;
                    PFB_CU(cudaMemcpyAsync(reinterpret_cast<unsigned char*>(ring) + (size_t)(k % frames) * frame_bytes,
                                           d_traj, frame_bytes, cudaMemcpyDeviceToHost, stream),
                           "download traj");
                }
                ++k;
            }
        }
        return settle_bins();
    }

    // Allocate every device buffer for p (reference src/sim.cu:159-232).
    int alloc(const pfb_params2d& prm, int dev) {
        p = prm;
        device = dev;
        N = p.num_cells;
        L = p.L;
        if (N < 1) return set_error(PFB_E_ARG, "num_cells must be positive");
        if (L < kMinSide) return set_error(PFB_E_ARG, "domain side %d is below %d", L, kMinSide);
        if (p.phi_storage < 0 || p.phi_storage > 2)
            return set_error(PFB_E_ARG, "phi_storage must be 0, 1 or 2");
        P = 32 * ((L + 31) / 32);
        s_words = (size_t)P * (size_t)L;
        PFB_CU(cudaSetDevice(device), "cudaSetDevice");
        const size_t pool = pool_bytes();
        PFB_CU(cudaMalloc(&d_phi[0], pool), "alloc phi");
        PFB_CU(cudaMalloc(&d_phi[1], pool), "alloc phi");
        PFB_CU(cudaMalloc(&d_S, 3 * s_words * sizeof(uint32_t)), "alloc S");
        PFB_CU(cudaMalloc(&d_cell, (size_t)N * sizeof(pfb_cell2d)), "alloc cells");
        PFB_CU(cudaMalloc(&d_cls, (size_t)N), "alloc classes");
        PFB_CU(cudaMalloc(&d_cursor, 2 * sizeof(unsigned long long)), "alloc cursor");
        PFB_CU(cudaMalloc(&d_step, 2 * sizeof(unsigned long long)), "alloc step");
        PFB_CU(cudaMalloc(&d_flags, PFB_FLAG_COUNT * sizeof(uint32_t)), "alloc flags");
        PFB_CU(cudaMalloc(&d_traj, (size_t)N * sizeof(pfb_traj_cell2d)), "alloc traj");
        PFB_CU(cudaMalloc(&d_cell_prev, (size_t)N * sizeof(pfb_cell2d)), "alloc cells");
        nbins_side = (L + (1 << kBinShift) - 1) >> kBinShift;
        PFB_CU(cudaMalloc(&d_bins, bin_words() * sizeof(unsigned long long)), "alloc bins");
        PFB_CU(cudaMalloc(&d_geo, 2 * (size_t)N * sizeof(int4)), "alloc bins");
        PFB_CU(cudaMalloc(&d_recounts, sizeof(unsigned int)), "alloc bins");
        PFB_CU(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "stream");
        PFB_CU(cudaMemsetAsync(d_recounts, 0, sizeof(unsigned int), stream), "clear bins");
        PFB_CU(cudaMemsetAsync(d_geo, 0, 2 * (size_t)N * sizeof(int4), stream), "clear bins");
        if (const int rc = reset_bins()) return rc;
        PFB_CU(cudaMemsetAsync(d_cursor, 0, 2 * sizeof(unsigned long long), stream), "memset");
        PFB_CU(cudaMemsetAsync(d_step, 0, 2 * sizeof(unsigned long long), stream), "memset");
        PFB_CU(cudaMemsetAsync(d_flags, 0, PFB_FLAG_COUNT * sizeof(uint32_t), stream), "memset");
        PFB_CU(cudaMemsetAsync(d_S, 0, 3 * s_words * sizeof(uint32_t), stream), "memset");
        return step2d_configure_device();
    }

    int set_state(const pfb_cell2d* cells, const float* phi, long long step) {
        if (!cells || !phi || step < 0) return set_error(PFB_E_ARG, "set_state: bad argument");
        PFB_CU(cudaSetDevice(device), "cudaSetDevice");
        drop_graph();
        steps_done = step;
        const int pin = (int)(step % 2), rot = (int)(step % 3);
        std::vector<pfb_cell2d> h((size_t)N);
        std::vector<uint8_t> hc((size_t)N);
        for (int i = 0; i < N; ++i) {
            h[(size_t)i] = cells[i];
            h[(size_t)i].cls_written[0] = cells[i].cls;
            h[(size_t)i].cls_written[1] = cells[i].cls;
            hc[(size_t)i] = cells[i].cls;
        }
        const size_t pool = pool_bytes();
        const size_t fwords = (size_t)N * kTileArea;
        PFB_CU(cudaMemcpyAsync(d_cell, h.data(), h.size() * sizeof(pfb_cell2d),
                               cudaMemcpyHostToDevice, stream), "upload cells");
        PFB_CU(cudaMemcpyAsync(d_cls, hc.data(), hc.size(), cudaMemcpyHostToDevice, stream),
               "upload classes");
        float* scan = nullptr;  // binary32 field the aggregate is built from
        if (p.phi_storage) {
            PFB_CU(cudaMalloc(&scan, fwords * sizeof(float)), "alloc staging field");
            PFB_CU(cudaMemcpyAsync(scan, phi, fwords * sizeof(float), cudaMemcpyHostToDevice, stream),
                   "upload phi");
            int rc = narrow_pool(scan, d_phi[pin], fwords, p.phi_storage, stream);
            if (!rc) rc = widen(pin, scan);
            if (rc) {
                cudaFree(scan);
                return rc;
            }
        } else {
            PFB_CU(cudaMemcpyAsync(d_phi[pin], phi, pool, cudaMemcpyHostToDevice, stream),
                   "upload phi");
        }
        PFB_CU(cudaMemsetAsync(d_phi[1 - pin], 0, pool, stream), "clear phi");
        const unsigned long long hs[2] = {
            (unsigned long long)(pin == 0 ? step : step + 1),
            (unsigned long long)(pin == 1 ? step : step + 1)};
        PFB_CU(cudaMemcpyAsync(d_step, hs, sizeof(hs), cudaMemcpyHostToDevice, stream), "upload step");
        PFB_CU(cudaMemsetAsync(d_cursor, 0, 2 * sizeof(unsigned long long), stream), "memset");
        if (const int rc2 = reset_bins()) return rc2;
        PFB_CU(cudaMemsetAsync(d_S, 0, 3 * s_words * sizeof(uint32_t), stream), "memset S");
        int rc = scatter_all2d(scan ? scan : (const float*)d_phi[pin], d_cell, d_cls,
                               d_S + (size_t)rot * s_words, N, L, P, d_flags, stream);
        const cudaError_t e = cudaStreamSynchronize(stream);
        cudaFree(scan);
        if (rc) return rc;
        PFB_CU(e, "set_state sync");
        return PFB_OK;
    }

    // Fresh start (reference src/sim.cu:308-370).
    int init_fresh(const float* cx, const float* cy) {
        if (!cx || !cy) return set_error(PFB_E_ARG, "centres are required");
        std::vector<pfb_cell2d> h((size_t)N);
        std::memset(h.data(), 0, h.size() * sizeof(pfb_cell2d));
        const unsigned long long pstream = p.polarity_seed ? p.polarity_seed : p.seed;
        const int n_cancer = (int)std::llround(p.cancer_fraction * (double)N);
        for (int i = 0; i < N; ++i) {
            pfb_cell2d& c = h[(size_t)i];
            c.global_id = i;
            c.gamma = (float)(i < n_cancer ? p.gamma_cancer : p.gamma_normal);
            c.v_A = (float)pfb_ic_v_A(i, p.seed, p.v_A, p.v_A_sigma);
            c.M_pf = (float)p.phase_field_mobility;
            c.R_tgt = (float)p.target_radius;
            c.theta = pfb_ic_theta(i, pstream);
            c.cls = 0;
            c.cls_written[0] = 0;
            c.cls_written[1] = 0;
        }
        std::vector<uint8_t> hc((size_t)N, 0);
        float *d_cx = nullptr, *d_cy = nullptr;
        PFB_CU(cudaMemcpyAsync(d_cell, h.data(), h.size() * sizeof(pfb_cell2d),
                               cudaMemcpyHostToDevice, stream), "upload cells");
        PFB_CU(cudaMemcpyAsync(d_cls, hc.data(), hc.size(), cudaMemcpyHostToDevice, stream),
               "upload classes");
        PFB_CU(cudaMalloc(&d_cx, (size_t)N * sizeof(float)), "alloc centres");
        PFB_CU(cudaMalloc(&d_cy, (size_t)N * sizeof(float)), "alloc centres");
        PFB_CU(cudaMemcpyAsync(d_cx, cx, (size_t)N * sizeof(float), cudaMemcpyHostToDevice, stream),
               "upload centres");
        PFB_CU(cudaMemcpyAsync(d_cy, cy, (size_t)N * sizeof(float), cudaMemcpyHostToDevice, stream),
               "upload centres");
        // 16-bit pools: seed binary32 tiles in temporaries, round them to
        // nearest into the pool and measure / scatter the stored values
        float* f0 = nullptr;
        float* f1 = nullptr;
        if (p.phi_storage) {
            PFB_CU(cudaMalloc(&f0, (size_t)N * kTileArea * sizeof(float)), "alloc staging field");
            PFB_CU(cudaMalloc(&f1, (size_t)N * kTileArea * sizeof(float)), "alloc staging field");
        }
        float* a0 = p.phi_storage ? f0 : (float*)d_phi[0];
        float* a1 = p.phi_storage ? f1 : (float*)d_phi[1];
        int rc = init_tiles2d(a0, a1, d_cell, d_cls, N, L, d_cx, d_cy,
                              (float)seed_radius(p.target_radius, p.lambda),
                              (float)iface_k(p.lambda), stream);
        if (!rc && p.phi_storage) {
            rc = narrow_pool(f0, d_phi[0], (size_t)N * kTileArea, p.phi_storage, stream);
            if (!rc) rc = narrow_pool(f1, d_phi[1], (size_t)N * kTileArea, p.phi_storage, stream);
            if (!rc) rc = widen(0, f0);
        }
        if (!rc) rc = init_moments2d(d_cell, d_cls, a0, N, stream);
        if (!rc) rc = scatter_all2d(a0, d_cell, d_cls, d_S, N, L, P, d_flags, stream);
        const cudaError_t e = cudaStreamSynchronize(stream);
        cudaFree(d_cx);
        cudaFree(d_cy);
        cudaFree(f0);
        cudaFree(f1);
        if (rc) return rc;
        PFB_CU(e, "init sync");
        steps_done = 0;
        return PFB_OK;
    }
};

namespace {
cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }
}  // namespace

extern "C" {

int pfb_step2d_configure(void) { return step2d_configure_device(); }

int pfb_step2d_grid(int num_cells, int cluster) {
    if (cluster == 0) cluster = kDefaultCluster;
    if (num_cells < 0 || (cluster != 2 && cluster != 4 && cluster != 8)) return PFB_E_ARG;
    return num_cells * cluster;
}

int pfb_step2d_launch(const pfb_step_args2d* args, int cluster, void* stream) {
    return step2d_launch(args, cluster, as_stream(stream));
}

int pfb_step2d_launch_ex(const pfb_step_args2d* args, int cluster, int variant, void* stream) {
    return step2d_launch_variant(args, cluster, variant, as_stream(stream));
}

int pfb_step2d_launch_observed(const pfb_step_args2d* args, int cluster, int observation,
                               void* stream) {
    return step2d_launch_observed(args, cluster, observation, as_stream(stream));
}

int pfb_velocity_moments2d(const pfb_step_args2d* args, pfb_moment_accum2d* out,
                           double physical_dt, void* stream) {
    if (!args) return set_error(PFB_E_ARG, "null step arguments");
    if (!(physical_dt > 0.0)) return set_error(PFB_E_ARG, "physical_dt must be positive");
    return velocity2d_observe(*args, out, physical_dt, as_stream(stream));
}

int pfb_sim2d_velocity_open(pfb_sim2d* s, const char* path, int spatial_stride,
                            long long dense_start, int reference) {
    if (!s) return set_error(PFB_E_ARG, "null system");
    if (s->vel) return set_error(PFB_E_STATE, "a velocity recorder is already open");
    if (s->p.phi_storage != 0)
        return set_error(PFB_E_CONFIG, "velocity observation needs binary32 phi pools");
    PFB_CU(cudaSetDevice(s->device), "cudaSetDevice");
    Velocity2D* v = velocity2d_create(path, s->N, s->p.dt, spatial_stride, dense_start, reference);
    if (!v) return PFB_E_ARG;
    const pfb_step_args2d a = s->args_for_slot((int)(s->steps_done % 6));
    const int rc = velocity2d_open(v, a, s->steps_done, s->stream);
    if (rc) {
        velocity2d_destroy(v);
        return rc;
    }
    s->vel = v;
    return PFB_OK;
}

int pfb_sim2d_velocity_capture(pfb_sim2d* s) {
    if (!s || !s->vel) return set_error(PFB_E_STATE, "no velocity recorder is open");
    PFB_CU(cudaSetDevice(s->device), "cudaSetDevice");
    const pfb_step_args2d a = s->args_for_slot((int)(s->steps_done % 6));
    return velocity2d_capture(s->vel, a, s->steps_done, s->stream);
}

long long pfb_sim2d_velocity_last_frame(const pfb_sim2d* s) {
    return s && s->vel ? velocity2d_last_frame(s->vel) : -1;
}

int pfb_sim2d_boundary_open(pfb_sim2d* s, const char* path, long long interval, int compress) {
    if (!s) return set_error(PFB_E_ARG, "null system");
    if (s->bnd) return set_error(PFB_E_STATE, "a boundary recorder is already open");
    if (s->p.phi_storage != 0)
        return set_error(PFB_E_CONFIG, "the boundary recorder needs binary32 phi pools");
    PFB_CU(cudaSetDevice(s->device), "cudaSetDevice");
    s->bnd = boundary2d_open(path, s->N, s->L, s->p.dt, s->p.tau, interval, compress);
    return s->bnd ? PFB_OK : PFB_E_ARG;
}

int pfb_sim2d_boundary_capture(pfb_sim2d* s) {
    if (!s || !s->bnd) return set_error(PFB_E_STATE, "no boundary recorder is open");
    PFB_CU(cudaSetDevice(s->device), "cudaSetDevice");
    return boundary2d_capture(s->bnd, s->d_phi[s->steps_done % 2], s->d_cell, s->stream,
                              s->steps_done, (double)s->steps_done * s->p.dt);
}

int pfb_sim2d_boundary_close(pfb_sim2d* s) {
    if (!s || !s->bnd) return set_error(PFB_E_STATE, "no boundary recorder is open");
    const int rc = boundary2d_close(s->bnd);
    s->bnd = nullptr;
    return rc;
}

int pfb_sim2d_verify(pfb_sim2d* s, double* max_rel_V, float* max_outside, uint32_t* max_S) {
    if (!s || !max_rel_V || !max_outside || !max_S) return set_error(PFB_E_ARG, "verify: null argument");
    if (s->p.phi_storage != 0) return set_error(PFB_E_CONFIG, "verify needs binary32 phi pools");
    PFB_CU(cudaSetDevice(s->device), "cudaSetDevice");
    double* d_v = nullptr;
    float* d_o = nullptr;
    uint32_t* d_m = nullptr;
    const size_t N = (size_t)s->N;
    int rc = PFB_OK;
    std::vector<double> v(N);
    std::vector<float> o(N);
    std::vector<pfb_cell2d> c(N);
    if (cudaMalloc(&d_v, N * sizeof(double)) != cudaSuccess || cudaMalloc(&d_o, N * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&d_m, sizeof(uint32_t)) != cudaSuccess || cudaMemsetAsync(d_m, 0, 4, s->stream) != cudaSuccess) {
        rc = set_error(PFB_E_CUDA, "verify: allocation failed");
    } else {
        const int pin = (int)(s->steps_done % 2), rot = (int)(s->steps_done % 3);
        rc = verify_cells2d(s->d_phi[pin], s->d_cell, s->d_cls, s->N, d_v, d_o, s->stream);
        if (!rc) rc = verify_S(s->d_S + (size_t)rot * s->s_words, s->s_words, d_m, s->stream);
        if (!rc && (cudaMemcpyAsync(v.data(), d_v, N * sizeof(double), cudaMemcpyDeviceToHost, s->stream) !=
                        cudaSuccess ||
                    cudaMemcpyAsync(o.data(), d_o, N * sizeof(float), cudaMemcpyDeviceToHost, s->stream) !=
                        cudaSuccess ||
                    cudaMemcpyAsync(c.data(), s->d_cell, N * sizeof(pfb_cell2d), cudaMemcpyDeviceToHost,
                                    s->stream) != cudaSuccess ||
                    cudaMemcpyAsync(max_S, d_m, 4, cudaMemcpyDeviceToHost, s->stream) != cudaSuccess ||
                    cudaStreamSynchronize(s->stream) != cudaSuccess))
            rc = set_error(PFB_E_CUDA, "verify: readback failed");
    }
    cudaFree(d_v);
    cudaFree(d_o);
    cudaFree(d_m);
    if (rc) return rc;
    double mr = 0.0;
    float mo = 0.0f;
    for (size_t i = 0; i < N; ++i) {
        const double den = std::max(1e-12, std::fabs(c[i].V));
        mr = std::max(mr, std::fabs(v[i] - c[i].V) / den);
        mo = std::max(mo, o[i]);
    }
    *max_rel_V = mr;
    *max_outside = mo;
    return PFB_OK;
}

int pfb_sim2d_velocity_close(pfb_sim2d* s) {
    if (!s || !s->vel) return set_error(PFB_E_STATE, "no velocity recorder is open");
    const int rc = velocity2d_close(s->vel);
    velocity2d_destroy(s->vel);
    s->vel = nullptr;
    return rc;
}

int pfb_init_tiles2d(float* phi_a, float* phi_b, pfb_cell2d* cell, const uint8_t* cls, int N,
                     int L, const float* seed_cx, const float* seed_cy, float radius_eff,
                     float kappa_iface, void* stream) {
    return init_tiles2d(phi_a, phi_b, cell, cls, N, L, seed_cx, seed_cy, radius_eff, kappa_iface,
                        as_stream(stream));
}

int pfb_init_moments2d(pfb_cell2d* cell, const uint8_t* cls, const float* phi, int N,
                       void* stream) {
    return init_moments2d(cell, cls, phi, N, as_stream(stream));
}

int pfb_scatter_all2d(const float* phi, const pfb_cell2d* cell, const uint8_t* cls, uint32_t* S,
                      int N, int L, int P, uint32_t* flags, void* stream) {
    return scatter_all2d(phi, cell, cls, S, N, L, P, flags, as_stream(stream));
}

int pfb_zero_u32(uint32_t* p, size_t n, void* stream) { return zero_u32(p, n, as_stream(stream)); }

int pfb_verify_cells2d(const float* phi, const pfb_cell2d* cell, const uint8_t* cls, int N,
                       double* out_V, float* out_outside_max, void* stream) {
    return verify_cells2d(phi, cell, cls, N, out_V, out_outside_max, as_stream(stream));
}

int pfb_verify_S(const uint32_t* S, size_t n, uint32_t* out_max, void* stream) {
    return verify_S(S, n, out_max, as_stream(stream));
}

int pfb_pack_traj2d(const pfb_cell2d* cell, const uint8_t* cls, pfb_traj_cell2d* out, int N,
                    int L, void* stream) {
    return pack_traj2d(cell, cls, out, N, L, as_stream(stream));
}

int pfb_device_status(unsigned* out, int clear) {
    unsigned a = 0, b = 0;
    int rc = step2d_read_status(&a, clear);
    if (!rc) rc = init2d_read_status(&b, clear);
    if (out) *out = a | (b << 2);
    return rc;
}

pfb_sim2d* pfb_sim2d_create(const pfb_params2d* p, const float* cx, const float* cy, int device) {
    clear_error();
    if (!p) {
        set_error(PFB_E_ARG, "null params");
        return nullptr;
    }
    pfb_sim2d* s = new (std::nothrow) pfb_sim2d();
    if (!s) {
        set_error(PFB_E_NOMEM, "host allocation failed");
        return nullptr;
    }
    if (s->alloc(*p, device) || s->init_fresh(cx, cy)) {
        delete s;
        return nullptr;
    }
    return s;
}

pfb_sim2d* pfb_sim2d_create_from_state(const pfb_params2d* p, const pfb_cell2d* cells,
                                       const float* phi, long long step, int device) {
    clear_error();
    if (!p) {
        set_error(PFB_E_ARG, "null params");
        return nullptr;
    }
    pfb_sim2d* s = new (std::nothrow) pfb_sim2d();
    if (!s) {
        set_error(PFB_E_NOMEM, "host allocation failed");
        return nullptr;
    }
    if (s->alloc(*p, device) || s->set_state(cells, phi, step)) {
        delete s;
        return nullptr;
    }
    return s;
}

void pfb_sim2d_destroy(pfb_sim2d* s) {
    if (s) {
        cudaSetDevice(s->device);
        delete s;
    }
}

int pfb_sim2d_set_cluster(pfb_sim2d* s, int cluster) {
    if (!s) return set_error(PFB_E_ARG, "null sim");
    if (cluster != 2 && cluster != 4 && cluster != 8) return set_error(PFB_E_CONFIG, "cluster must be 2, 4 or 8");
    if (cluster == 8 && s->p.phi_storage)
        return set_error(PFB_E_CONFIG, "16-bit phi pools run with clusters of 2 or 4");
    if (cluster != s->cluster) s->drop_graph();
    s->cluster = cluster;
    return PFB_OK;
}

int pfb_sim2d_set_variant(pfb_sim2d* s, int variant) {
    if (!s) return set_error(PFB_E_ARG, "null sim");
    if (variant < 0 || variant > 2) return set_error(PFB_E_CONFIG, "unknown kernel variant");
    if (variant != s->variant) s->drop_graph();
    s->variant = variant;
    return PFB_OK;
}

int pfb_sim2d_scatter_recounts(pfb_sim2d* s, unsigned int* out) {
    if (!s || !out) return set_error(PFB_E_ARG, "scatter_recounts: null argument");
    PFB_CU(cudaSetDevice(s->device), "cudaSetDevice");
    PFB_CU(cudaMemcpyAsync(out, s->d_recounts, sizeof(unsigned int), cudaMemcpyDeviceToHost,
                           s->stream),
           "read recounts");
    PFB_CU(cudaStreamSynchronize(s->stream), "read recounts");
    return PFB_OK;
}

int pfb_sim2d_set_graph(pfb_sim2d* s, int use_graph) {
    if (!s) return set_error(PFB_E_ARG, "null sim");
    s->use_graph = use_graph != 0;
    if (!s->use_graph) s->drop_graph();
    return PFB_OK;
}

int pfb_sim2d_set_visit_order(pfb_sim2d* s, int order) {
    if (!s) return set_error(PFB_E_ARG, "null sim");
    if (order != PFB_VISIT_LAUNCH && order != PFB_VISIT_MORTON) return set_error(PFB_E_ARG, "unknown visit order");
    PFB_CU(cudaSetDevice(s->device), "cudaSetDevice");
    if (order == PFB_VISIT_LAUNCH) {
        if (s->d_perm) {
            s->drop_graph();
            PFB_CU(cudaStreamSynchronize(s->stream), "sync");
            cudaFree(s->d_perm);
            s->d_perm = nullptr;
        }
        return PFB_OK;
    }
    if (s->d_perm) return PFB_OK;
    const int cap = visit_order2d_capacity();
    if (s->N > cap) {
        size_t m = 1;
        while (m < (size_t)s->N) m <<= 1;
        return set_error(PFB_E_CONFIG,
                         "Morton order needs %.1f KB of shared memory for N=%d; the sort holds at most %d cells",
                         (double)(m * sizeof(unsigned long long)) / 1024.0, s->N, cap);
    }
    PFB_CU(visit_order2d_prepare(s->N), "visit order attribute");
    PFB_CU(cudaMalloc(&s->d_perm, (size_t)s->N * sizeof(uint32_t)), "alloc visit order");
    // sorted now, so that a start at any step finds a valid order
    if (cudaError_t e = visit_order2d_launch(s->d_cell, s->d_perm, s->N, s->L, s->stream)) {
        cudaFree(s->d_perm);
        s->d_perm = nullptr;
        PFB_CU(e, "visit order");
    }
    s->drop_graph();
    return PFB_OK;
}

int pfb_sim2d_visit_order(pfb_sim2d* s, uint32_t* out) {
    if (!s || !out) return set_error(PFB_E_ARG, "visit_order: bad argument");
    if (!s->d_perm) {
        for (int i = 0; i < s->N; ++i) out[i] = (uint32_t)i;
        return PFB_OK;
    }
    PFB_CU(cudaSetDevice(s->device), "cudaSetDevice");
    PFB_CU(cudaMemcpyAsync(out, s->d_perm, (size_t)s->N * sizeof(uint32_t), cudaMemcpyDeviceToHost, s->stream),
           "visit order copy");
    PFB_CU(cudaStreamSynchronize(s->stream), "sync");
    return PFB_OK;
}

int pfb_sim2d_advance(pfb_sim2d* s, long long steps) {
    if (!s || steps < 0) return set_error(PFB_E_ARG, "advance: bad argument");
    PFB_CU(cudaSetDevice(s->device), "cudaSetDevice");
    return s->advance(steps);
}

int pfb_sim2d_sync(pfb_sim2d* s) {
    if (!s) return set_error(PFB_E_ARG, "null sim");
    PFB_CU(cudaStreamSynchronize(s->stream), "sync");
    return PFB_OK;
}

long long pfb_sim2d_step(const pfb_sim2d* s) { return s ? s->steps_done : -1; }
int pfb_sim2d_side(const pfb_sim2d* s) { return s ? s->L : -1; }
int pfb_sim2d_pitch(const pfb_sim2d* s) { return s ? s->P : -1; }
int pfb_sim2d_num_cells(const pfb_sim2d* s) { return s ? s->N : -1; }

int pfb_sim2d_get_cells(pfb_sim2d* s, pfb_cell2d* out) {
    if (!s || !out) return set_error(PFB_E_ARG, "get_cells: null");
    PFB_CU(cudaMemcpyAsync(out, s->d_cell, (size_t)s->N * sizeof(pfb_cell2d),
                           cudaMemcpyDeviceToHost, s->stream), "download cells");
    PFB_CU(cudaStreamSynchronize(s->stream), "sync");
    return PFB_OK;
}

int pfb_sim2d_get_phi(pfb_sim2d* s, float* out) {
    if (!s || !out) return set_error(PFB_E_ARG, "get_phi: null");
    const int pin = (int)(s->steps_done % 2);
    const size_t bytes = (size_t)s->N * kTileArea * sizeof(float);
    if (s->p.phi_storage) {
        float* tmp = nullptr;
        PFB_CU(cudaMalloc(&tmp, bytes), "alloc staging field");
        int rc = s->widen(pin, tmp);
        const cudaError_t e = rc ? cudaSuccess
                                 : cudaMemcpyAsync(out, tmp, bytes, cudaMemcpyDeviceToHost, s->stream);
        const cudaError_t e2 = cudaStreamSynchronize(s->stream);
        cudaFree(tmp);
        if (rc) return rc;
        PFB_CU(e, "download phi");
        PFB_CU(e2, "sync");
        return PFB_OK;
    }
    PFB_CU(cudaMemcpyAsync(out, s->d_phi[pin], bytes, cudaMemcpyDeviceToHost, s->stream),
           "download phi");
    PFB_CU(cudaStreamSynchronize(s->stream), "sync");
    return PFB_OK;
}

int pfb_sim2d_get_S(pfb_sim2d* s, uint32_t* out) {
    if (!s || !out) return set_error(PFB_E_ARG, "get_S: null");
    const int rot = (int)(s->steps_done % 3);
    PFB_CU(cudaMemcpyAsync(out, s->d_S + (size_t)rot * s->s_words, s->s_words * sizeof(uint32_t),
                           cudaMemcpyDeviceToHost, s->stream), "download S");
    PFB_CU(cudaStreamSynchronize(s->stream), "sync");
    return PFB_OK;
}

int pfb_sim2d_get_flags(pfb_sim2d* s, uint32_t* out) {
    if (!s || !out) return set_error(PFB_E_ARG, "get_flags: null");
    PFB_CU(cudaMemcpyAsync(out, s->d_flags, PFB_FLAG_COUNT * sizeof(uint32_t),
                           cudaMemcpyDeviceToHost, s->stream), "download flags");
    PFB_CU(cudaStreamSynchronize(s->stream), "sync");
    return PFB_OK;
}

int pfb_sim2d_save(pfb_sim2d* s) {
    if (!s) return set_error(PFB_E_ARG, "null system");
    return s->save();
}

int pfb_sim2d_restore(pfb_sim2d* s) {
    if (!s) return set_error(PFB_E_ARG, "null system");
    return s->restore();
}

int pfb_sim2d_set_state(pfb_sim2d* s, const pfb_cell2d* cells, const float* phi, long long step) {
    if (!s) return set_error(PFB_E_ARG, "null sim");
    return s->set_state(cells, phi, step);
}

int pfb_sim2d_pack_traj(pfb_sim2d* s, pfb_traj_cell2d* out) {
    if (!s || !out) return set_error(PFB_E_ARG, "pack_traj: null");
    int rc = pack_traj2d(s->d_cell, s->d_cls, s->d_traj, s->N, s->L, s->stream);
    if (rc) return rc;
    PFB_CU(cudaMemcpyAsync(out, s->d_traj, (size_t)s->N * sizeof(pfb_traj_cell2d),
                           cudaMemcpyDeviceToHost, s->stream), "download traj");
    PFB_CU(cudaStreamSynchronize(s->stream), "sync");
    return PFB_OK;
}

int pfb_sim2d_advance_record(pfb_sim2d* s, long long steps, int every, pfb_traj_cell2d* ring,
                             int frames) {
    if (!s || steps < 0 || every < 1 || !ring || frames < 1)
        return set_error(PFB_E_ARG, "advance_record: bad argument");
    PFB_CU(cudaSetDevice(s->device), "cudaSetDevice");
    return s->advance_record(steps, every, ring, frames);
}

int pfb_sim2d_bench(pfb_sim2d* s, int warmup, int steps, double* ms_per_step) {
    if (!s || warmup < 0 || steps < 1 || !ms_per_step) return set_error(PFB_E_ARG, "bench: bad argument");
    PFB_CU(cudaSetDevice(s->device), "cudaSetDevice");
    int rc = s->advance(warmup);
    if (rc) return rc;
    if (s->use_graph) {
        const long long align = (6 - s->steps_done % 6) % 6;
        rc = s->advance(align);
        if (rc) return rc;
    }
    PFB_CU(cudaStreamSynchronize(s->stream), "sync");
    cudaEvent_t e0, e1;
    PFB_CU(cudaEventCreate(&e0), "event");
    PFB_CU(cudaEventCreate(&e1), "event");
    cudaEventRecord(e0, s->stream);
    rc = s->advance(steps);
    cudaEventRecord(e1, s->stream);
    const cudaError_t e = cudaEventSynchronize(e1);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    PFB_CU(e, "bench sync");
    *ms_per_step = (double)ms / (double)steps;
    return PFB_OK;
}

int pfb_sim2d_step_args(pfb_sim2d* s, pfb_step_args2d* out) {
    if (!s || !out) return set_error(PFB_E_ARG, "step_args: null");
    *out = s->args_for_slot((int)(s->steps_done % 6));
    return PFB_OK;
}

void* pfb_sim2d_stream(pfb_sim2d* s) { return s ? (void*)s->stream : nullptr; }

}  // extern "C"

// ---------------------------------------------------------------------------
// Batched ensemble: R independent 2D systems of any size advanced by one
// launch per step (k_step2d_batch), six steps per CUDA graph. Each system
// keeps its own buffers, slots and device step counters (a pfb_sim2d); the
// ensemble owns the batch argument tables and its stream.
// ---------------------------------------------------------------------------
struct pfb_ens2d {
    std::vector<pfb_sim2d*> sims;
    std::vector<int> order;  // launch order of the systems (largest first)
    int device = 0;
    int cluster = kDefaultCluster;
    int storage = 0;  // phi pool type shared by every system
    long long steps_done = 0;
    cudaStream_t stream = nullptr;
    pfb_step_args2d* d_args = nullptr;  // 6 slots x R records
    int* d_start = nullptr;             // R + 1 block offsets
    int total_blocks = 0;
    bool tables_ready = false;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    // trajectory recording: sources of the batched pack (system order), the
    // ring header, a device frame for pageable rings, record graphs
    // [every - 1][phase] as pfb_sim2d's
    TrajSource2D* d_src = nullptr;
    TrajRing2D* d_ring = nullptr;
    pfb_traj_cell2d* d_frame = nullptr;
    int total_cells = 0;
    cudaGraphExec_t rec_exec[6][6] = {};

    ~pfb_ens2d() {
        drop_graph();
        if (stream) cudaStreamDestroy(stream);
        cudaFree(d_args);
        cudaFree(d_start);
        cudaFree(d_src);
        cudaFree(d_ring);
        cudaFree(d_frame);
        for (pfb_sim2d* s : sims) delete s;
    }

    int R() const { return (int)sims.size(); }

    void drop_graph() {
        if (graph_exec) cudaGraphExecDestroy(graph_exec);
        if (graph) cudaGraphDestroy(graph);
        graph_exec = nullptr;
        graph = nullptr;
        for (auto& row : rec_exec)
            for (cudaGraphExec_t& e : row) {
                if (e) cudaGraphExecDestroy(e);
                e = nullptr;
            }
    }

    // The pack sources in system order (buffers are fixed for the life of
    // the ensemble).
    int build_sources() {
        std::vector<TrajSource2D> h((size_t)R());
        int off = 0;
        for (int r = 0; r < R(); ++r) {
            h[(size_t)r] = TrajSource2D{sims[(size_t)r]->d_cell, sims[(size_t)r]->d_cls, sims[(size_t)r]->L, off};
            off += sims[(size_t)r]->N;
        }
        total_cells = off;
        PFB_CU(cudaMalloc(&d_src, h.size() * sizeof(TrajSource2D)), "alloc sources");
        PFB_CU(cudaMalloc(&d_ring, sizeof(TrajRing2D)), "alloc ring");
        PFB_CU(cudaMalloc(&d_frame, (size_t)total_cells * sizeof(pfb_traj_cell2d)), "alloc frame");
        PFB_CU(cudaMemcpyAsync(d_src, h.data(), h.size() * sizeof(TrajSource2D), cudaMemcpyHostToDevice,
                               stream),
               "upload sources");
        PFB_CU(cudaStreamSynchronize(stream), "sources");
        return PFB_OK;
    }

    int pack() { return pack_traj2d_ring_batch(d_src, R(), total_cells, d_ring, stream); }

    int build_record_graph(int every, int phase) {
        PFB_CU(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal), "begin capture");
        int rc = PFB_OK;
        for (int s = 0; s < 6 && rc == PFB_OK; ++s) {
            rc = launch_slot(s);
            if (rc == PFB_OK && (phase + s + 1) % every == 0) rc = pack();
        }
        cudaGraph_t g = nullptr;
        const cudaError_t e = cudaStreamEndCapture(stream, &g);
        if (rc != PFB_OK) {
            if (g) cudaGraphDestroy(g);
            return rc;
        }
        PFB_CU(e, "end capture");
        const cudaError_t ie = cudaGraphInstantiateWithFlags(&rec_exec[every - 1][phase], g, 0);
        cudaGraphDestroy(g);
        PFB_CU(ie, "graph instantiate");
        return PFB_OK;
    }

    // `steps` steps with every system's trajectory records of every
    // `every`-th step in ring frame k % frames (frames x total_cells records,
    // system r after the earlier systems' cells).
    int advance_record(long long steps, int every, pfb_traj_cell2d* ring, int frames) {
        if (!tables_ready) {
            if (const int rc = build_tables()) return rc;
        }
        if (!d_src) {
            if (const int rc = build_sources()) return rc;
        }
        const size_t frame_bytes = (size_t)total_cells * sizeof(pfb_traj_cell2d);
        pfb_traj_cell2d* dring = nullptr;
        cudaPointerAttributes at{};
        if (cudaPointerGetAttributes(&at, ring) == cudaSuccess && at.type == cudaMemoryTypeHost &&
            at.devicePointer && !((uintptr_t)at.devicePointer & 15u))
            dring = static_cast<pfb_traj_cell2d*>(at.devicePointer);
        (void)cudaGetLastError();  // an unregistered pointer is not an error here
        if (const int rc = ring_begin2d(d_ring, dring ? dring : d_frame, dring ? frames : 1, stream)) return rc;
        const bool rec_graph = dring && 6 % every == 0;
        long long done = 0, k = 0;
        while (done < steps) {
            const bool aligned = steps_done % 6 == 0 && steps - done >= 6;
            if (rec_graph && aligned) {
                const int phase = (int)(done % every);
                if (!rec_exec[every - 1][phase]) {
                    if (const int rc = build_record_graph(every, phase)) return rc;
                }
                PFB_CU(cudaGraphLaunch(rec_exec[every - 1][phase], stream), "graph launch");
                steps_done += 6;
                done += 6;
                continue;
            }
            const long long due = (done / every + 1) * every;
            if (aligned && due >= done + 6) {
                if (!graph_exec) {
                    if (const int rc = build_graph()) return rc;
                }
                PFB_CU(cudaGraphLaunch(graph_exec, stream), "graph launch");
                steps_done += 6;
                done += 6;
            } else {
                if (const int rc = launch_slot((int)(steps_done % 6))) return rc;
                steps_done += 1;
                done += 1;
            }
            if (done % every == 0) {
                if (const int rc = pack()) return rc;
                if (!dring)
                    PFB_CU(cudaMemcpyAsync(reinterpret_cast<unsigned char*>(ring) + (size_t)(k % frames) * frame_bytes,
                                           d_frame, frame_bytes, cudaMemcpyDeviceToHost, stream),
                           "download traj");
                ++k;
            }
        }
        for (pfb_sim2d* s : sims) s->steps_done = steps_done;
        return PFB_OK;
    }

    // Argument tables for the six slots and the CTA offsets for `cluster`.
    int build_tables() {
        drop_graph();
        const int R_ = R();
        std::vector<pfb_step_args2d> h((size_t)6 * R_);
        std::vector<int> start((size_t)R_ + 1, 0);
        for (int i = 0; i < R_; ++i) {
            const pfb_sim2d* s = sims[(size_t)order[(size_t)i]];
            for (int slot = 0; slot < 6; ++slot) h[(size_t)slot * R_ + i] = s->args_for_slot(slot);
            start[(size_t)i + 1] = start[(size_t)i] + s->N * cluster;
        }
        total_blocks = start[(size_t)R_];
        if (!d_args) PFB_CU(cudaMalloc(&d_args, h.size() * sizeof(pfb_step_args2d)), "alloc args");
        if (!d_start) PFB_CU(cudaMalloc(&d_start, start.size() * sizeof(int)), "alloc offsets");
        PFB_CU(cudaMemcpyAsync(d_args, h.data(), h.size() * sizeof(pfb_step_args2d),
                               cudaMemcpyHostToDevice, stream), "upload args");
        PFB_CU(cudaMemcpyAsync(d_start, start.data(), start.size() * sizeof(int),
                               cudaMemcpyHostToDevice, stream), "upload offsets");
        PFB_CU(cudaStreamSynchronize(stream), "tables");
        tables_ready = true;
        return PFB_OK;
    }

    int launch_slot(int slot) {
        return step2d_launch_batch(d_args + (size_t)slot * R(), d_start, R(), total_blocks, cluster,
                                   storage, stream);
    }

    int build_graph() {
        drop_graph();
        PFB_CU(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal), "begin capture");
        int rc = PFB_OK;
        for (int s = 0; s < 6 && rc == PFB_OK; ++s) rc = launch_slot(s);
        cudaGraph_t g = nullptr;
        const cudaError_t e = cudaStreamEndCapture(stream, &g);
        if (rc != PFB_OK) {
            if (g) cudaGraphDestroy(g);
            return rc;
        }
        PFB_CU(e, "end capture");
        graph = g;
        PFB_CU(cudaGraphInstantiateWithFlags(&graph_exec, graph, 0), "graph instantiate");
        return PFB_OK;
    }

    int advance(long long steps) {
        if (!tables_ready) {
            const int rc = build_tables();
            if (rc) return rc;
        }
        while (steps > 0) {
            if (steps_done % 6 == 0 && steps >= 6) {
                if (!graph_exec) {
                    const int rc = build_graph();
                    if (rc) return rc;
                }
                PFB_CU(cudaGraphLaunch(graph_exec, stream), "graph launch");
                steps_done += 6;
                steps -= 6;
            } else {
                const int rc = launch_slot((int)(steps_done % 6));
                if (rc) return rc;
                steps_done += 1;
                steps -= 1;
            }
        }
        for (pfb_sim2d* s : sims) s->steps_done = steps_done;
        return PFB_OK;
    }

    // The same steps with one launch per system (the replicas-one-at-a-time
    // baseline the batch is measured against).
    int advance_serial(long long steps) {
        for (long long k = 0; k < steps; ++k) {
            const int slot = (int)(steps_done % 6);
            for (pfb_sim2d* s : sims) {
                const pfb_step_args2d a = s->args_for_slot(slot);
                const int rc = step2d_launch_storage(&a, cluster, 0, storage, stream);
                if (rc) return rc;
            }
            ++steps_done;
        }
        for (pfb_sim2d* s : sims) s->steps_done = steps_done;
        return PFB_OK;
    }
};

extern "C" {

pfb_ens2d* pfb_ens2d_create(int R, const pfb_params2d* params, const float* const* cx,
                            const float* const* cy, int device) {
    clear_error();
    if (R <= 0 || !params || !cx || !cy) {
        set_error(PFB_E_ARG, "ensemble needs R > 0 systems with parameters and centres");
        return nullptr;
    }
    pfb_ens2d* e = new (std::nothrow) pfb_ens2d();
    if (!e) {
        set_error(PFB_E_NOMEM, "host allocation failed");
        return nullptr;
    }
    e->device = device;
    e->storage = params[0].phi_storage;
    for (int r = 0; r < R; ++r) {
        if (params[r].phi_storage != e->storage) {
            set_error(PFB_E_CONFIG, "every system of an ensemble needs the same phi_storage");
            delete e;
            return nullptr;
        }
        pfb_sim2d* s = pfb_sim2d_create(&params[r], cx[r], cy[r], device);
        if (!s) {
            delete e;
            return nullptr;
        }
        s->use_graph = false;
        e->sims.push_back(s);
    }
    e->order.resize((size_t)R);
    for (int r = 0; r < R; ++r) e->order[(size_t)r] = r;
    // largest systems first: their CTAs start in the first wave
    std::stable_sort(e->order.begin(), e->order.end(),
                     [e](int a, int b) { return e->sims[(size_t)a]->N > e->sims[(size_t)b]->N; });
    if (cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking) != cudaSuccess) {
        set_error(PFB_E_CUDA, "stream creation failed");
        delete e;
        return nullptr;
    }
    return e;
}

void pfb_ens2d_destroy(pfb_ens2d* e) { delete e; }

int pfb_ens2d_num_systems(const pfb_ens2d* e) { return e ? e->R() : -1; }

int pfb_ens2d_set_cluster(pfb_ens2d* e, int cluster) {
    if (!e) return set_error(PFB_E_ARG, "null ensemble");
    if (cluster == 0) cluster = kDefaultCluster;
    if (cluster != 2 && cluster != 4 && cluster != 8)
        return set_error(PFB_E_CONFIG, "cluster must be 2, 4 or 8");
    if (cluster == 8 && e->storage)
        return set_error(PFB_E_CONFIG, "16-bit phi pools run with clusters of 2 or 4");
    if (cluster != e->cluster) {
        e->cluster = cluster;
        e->tables_ready = false;
        e->drop_graph();
    }
    return PFB_OK;
}

int pfb_ens2d_advance(pfb_ens2d* e, int steps) {
    if (!e || steps < 0) return set_error(PFB_E_ARG, "advance: bad argument");
    PFB_CU(cudaSetDevice(e->device), "cudaSetDevice");
    return e->advance(steps);
}

void* pfb_ens2d_stream(pfb_ens2d* e) { return e ? (void*)e->stream : nullptr; }

int pfb_ens2d_advance_record(pfb_ens2d* e, long long steps, int every, pfb_traj_cell2d* ring, int frames) {
    if (!e || steps < 0 || every < 1 || !ring || frames < 1)
        return set_error(PFB_E_ARG, "advance_record: bad argument");
    PFB_CU(cudaSetDevice(e->device), "cudaSetDevice");
    return e->advance_record(steps, every, ring, frames);
}

int pfb_ens2d_advance_serial(pfb_ens2d* e, int steps) {
    if (!e || steps < 0) return set_error(PFB_E_ARG, "advance: bad argument");
    PFB_CU(cudaSetDevice(e->device), "cudaSetDevice");
    return e->advance_serial(steps);
}

int pfb_ens2d_sync(pfb_ens2d* e) {
    if (!e) return set_error(PFB_E_ARG, "null ensemble");
    PFB_CU(cudaStreamSynchronize(e->stream), "sync");
    return PFB_OK;
}

long long pfb_ens2d_step(const pfb_ens2d* e) { return e ? e->steps_done : -1; }

pfb_sim2d* pfb_ens2d_system(pfb_ens2d* e, int r) {
    if (!e || r < 0 || r >= e->R()) {
        set_error(PFB_E_ARG, "system index out of range");
        return nullptr;
    }
    if (cudaStreamSynchronize(e->stream) != cudaSuccess) {
        set_error(PFB_E_CUDA, "sync");
        return nullptr;
    }
    return e->sims[(size_t)r];
}

// Device time of `steps` steps after `warmup`, in ms per step; serial != 0
// launches the systems one at a time instead of in one batch.
int pfb_ens2d_bench(pfb_ens2d* e, int warmup, int steps, int serial, double* ms_per_step) {
    if (!e || warmup < 0 || steps < 1 || !ms_per_step) return set_error(PFB_E_ARG, "bench: bad argument");
    PFB_CU(cudaSetDevice(e->device), "cudaSetDevice");
    int rc = serial ? e->advance_serial(warmup) : e->advance(warmup);
    if (rc) return rc;
    if (!serial) {
        rc = e->advance((6 - e->steps_done % 6) % 6);
        if (rc) return rc;
    }
    PFB_CU(cudaStreamSynchronize(e->stream), "sync");
    cudaEvent_t e0, e1;
    PFB_CU(cudaEventCreate(&e0), "event");
    PFB_CU(cudaEventCreate(&e1), "event");
    cudaEventRecord(e0, e->stream);
    rc = serial ? e->advance_serial(steps) : e->advance(steps);
    cudaEventRecord(e1, e->stream);
    const cudaError_t err = cudaEventSynchronize(e1);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    PFB_CU(err, "bench sync");
    *ms_per_step = (double)ms / (double)steps;
    return PFB_OK;
}

// Time a few steps with each cluster size and keep the fastest (the
// ensemble's autotuner); writes the chosen size.
int pfb_ens2d_autotune(pfb_ens2d* e, int steps, int* chosen) {
    if (!e || steps < 1) return set_error(PFB_E_ARG, "autotune: bad argument");
    double best = 0.0;
    int best_k = e->cluster;
    const int ks[3] = {2, 4, 8};
    for (int k : ks) {
        if (k == 8 && e->storage) continue;
        int rc = pfb_ens2d_set_cluster(e, k);
        if (rc) return rc;
        double ms = 0.0;
        rc = pfb_ens2d_bench(e, 6, steps, 0, &ms);
        if (rc) return rc;
        if (best == 0.0 || ms < best) {
            best = ms;
            best_k = k;
        }
    }
    if (chosen) *chosen = best_k;
    return pfb_ens2d_set_cluster(e, best_k);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Device-side access for the relaxation tools (residual, surrogate jump):
// the current pool, the previous one, the cell records and the aggregate.
// ---------------------------------------------------------------------------
namespace pfb {

int sim2d_view(pfb_sim2d* s, Sim2DView* v) {
    if (!s || !v) return set_error(PFB_E_ARG, "sim2d_view: null argument");
    const int pin = (int)(s->steps_done % 2), rot = (int)(s->steps_done % 3);
    v->phi_cur = s->d_phi[pin];
    v->phi_prev = s->d_phi[1 - pin];
    v->cells = s->d_cell;
    v->cells_prev = s->d_cell_prev;
    v->cls = s->d_cls;
    v->S_cur = s->d_S + (size_t)rot * s->s_words;
    v->N = s->N;
    v->L = s->L;
    v->P = s->P;
    v->dt = s->p.dt;
    v->storage = s->p.phi_storage;
    v->stream = s->stream;
    v->step = s->steps_done;
    v->device = s->device;
    return PFB_OK;
}

// After the current binary32 pool was edited on the device: recompute the
// cells' moments and support from it and rebuild the current aggregate slot
// (the next slot, the following step's scatter target, is cleared too).
int sim2d_rebuild(pfb_sim2d* s) {
    if (!s) return set_error(PFB_E_ARG, "sim2d_rebuild: null system");
    if (s->p.phi_storage) return set_error(PFB_E_CONFIG, "rebuild needs binary32 pools");
    PFB_CU(cudaSetDevice(s->device), "cudaSetDevice");
    s->drop_graph();
    const int pin = (int)(s->steps_done % 2), rot = (int)(s->steps_done % 3);
    int rc = init_moments2d(s->d_cell, s->d_cls, s->d_phi[pin], s->N, s->stream);
    if (rc) return rc;
    PFB_CU(cudaMemsetAsync(s->d_S + (size_t)rot * s->s_words, 0, s->s_words * sizeof(uint32_t),
                           s->stream), "clear S");
    PFB_CU(cudaMemsetAsync(s->d_S + (size_t)((rot + 1) % 3) * s->s_words, 0,
                           s->s_words * sizeof(uint32_t), s->stream), "clear S");
    return scatter_all2d(s->d_phi[pin], s->d_cell, s->d_cls, s->d_S + (size_t)rot * s->s_words, s->N,
                         s->L, s->P, s->d_flags, s->stream);
}

// One step with the cell records saved first (for a residual between the two
// pools).
int sim2d_step_keep_prev(pfb_sim2d* s) {
    if (!s) return set_error(PFB_E_ARG, "sim2d_step_keep_prev: null system");
    PFB_CU(cudaSetDevice(s->device), "cudaSetDevice");
    PFB_CU(cudaMemcpyAsync(s->d_cell_prev, s->d_cell, (size_t)s->N * sizeof(pfb_cell2d),
                           cudaMemcpyDeviceToDevice, s->stream), "save cells");
    const int rc = s->launch_one((int)(s->steps_done % 6));
    if (rc) return rc;
    s->steps_done += 1;
    return s->settle_bins();
}

}  // namespace pfb
