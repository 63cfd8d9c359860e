// ORACLE -- test infrastructure only. A C-ABI shim around the reference's own
// 2D step kernel, compiled in place from the reference sources by
// oracle/Makefile into oracle/_ref/libref2d.so. GPU parity tests run it on the
// same device buffers as the product kernel (the step-argument record is
// byte-identical), so this is the reference itself, built for sm_100a.
//
// Binds (reference include/kernels.cuh:185-225):
//   pf::configure_k_step_smem, pf::k_step_grid, pf::launch_step,
//   pf::k_init_tiles, pf::k_init_moments, pf::k_scatter_all;
// and the host-side fresh-start draws pf::ic_theta, pf::ic_v_A (:146-172),
// which pin the oracle's restatement of them (no device needed).
#include <cstdio>

#include "kernels.cuh"

static_assert(sizeof(pf::StepArgs) == 216, "StepArgs layout");
static_assert(sizeof(pf::CellState) == 192, "CellState layout");

extern "C" {

int ref2d_configure(void) {
    pf::configure_k_step_smem();
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

int ref2d_grid(int device) { return pf::k_step_grid(device); }

int ref2d_launch_step(const void* args, int grid, void* stream) {
    static int configured = 0;
    if (!configured) {
        pf::configure_k_step_smem();
        configured = 1;
    }
    pf::launch_step(*static_cast<const pf::StepArgs*>(args), grid,
                    static_cast<cudaStream_t>(stream), nullptr, 0, 0.0f);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        std::fprintf(stderr, "ref2d_launch_step: %s\n", cudaGetErrorString(e));
        return -1;
    }
    return 0;
}

int ref2d_init_tiles(float* phi_a, float* phi_b, void* cell, const uint8_t* cls, int N, int L,
                     const float* cx, const float* cy, float radius_eff, float kappa_iface,
                     void* stream) {
    pf::k_init_tiles<<<N, 256, 0, static_cast<cudaStream_t>(stream)>>>(
        phi_a, phi_b, static_cast<pf::CellState*>(cell), cls, N, L, cx, cy, radius_eff,
        kappa_iface);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

int ref2d_init_moments(void* cell, const uint8_t* cls, const float* phi, int N, void* stream) {
    pf::k_init_moments<<<N, pf::kBlockThreads, 0, static_cast<cudaStream_t>(stream)>>>(
        static_cast<pf::CellState*>(cell), cls, phi, N);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

int ref2d_scatter_all(const float* phi, const void* cell, const uint8_t* cls, uint32_t* S, int N,
                      int L, int P, uint32_t* flags, void* stream) {
    pf::k_scatter_all<<<N, 256, 0, static_cast<cudaStream_t>(stream)>>>(
        phi, static_cast<const pf::CellState*>(cell), cls, S, N, L, P, flags);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

float ref2d_ic_theta(int32_t gid, unsigned long long stream) { return pf::ic_theta(gid, stream); }

double ref2d_ic_v_A(int32_t gid, unsigned long long seed, double v_A, double sigma) {
    return pf::ic_v_A(gid, seed, v_A, sigma);
}

}  // extern "C"
